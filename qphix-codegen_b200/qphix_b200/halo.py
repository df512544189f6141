"""T-slab domain decomposition of the dslash over ranks (one GPU per rank).

Each rank holds a local lattice of nt time slices; rank r owns global slices
[r*nt, (r+1)*nt).  One application of an operator on checkerboard cb is

  1. face_proj_dir (dir 7 and 6): project the t = nt-1 and t = 0 sites of psi
     for the forward / backward neighbour (codegen/dslash.cc:433-458);
  2. exchange the two face buffers with ranks r+1 and r-1;
  3. body kernel with accumulate[6] = accumulate[7] = 0: every hop except
     the ones that leave the slab (this overlaps step 2);
  4. face_*finish_dir (dir 6 and 7): add the received faces
     (codegen/dslash.cc:463-553).

The face kernels of the reference subtract beta*hop for Wilson and twisted
mass and add beta*A*hop for clover / TM clover (dslash_common.cc:1975-1981),
so each (family, kernel) pair maps to one face kind and a sign of beta (see
`face_kind`).  The time-boundary factor multiplies the beta of the faces that
cross the global t edge (rank 0 backward, last rank forward).

The compute steps are delegated to a `kernels` object (GPU kernels through
the C-ABI, or the CPU oracle in the tests) and the exchange to `TComm`, so the
same orchestration runs over NCCL on GPUs and over gloo on CPU.

`TSlabEvenOdd` composes two such applications into the even-odd operator
Mhat (the composition of qb200_schur_apply), and `cg` solves Mhat^dag Mhat
x = Mhat^dag b over the slabs: vectors stay local, each inner product is a
local FP64 sum followed by an all-reduce of the FP64 scalar.
"""
import math

import torch
import torch.distributed as dist

from .lattice import Geometry


def face_kind(family, kernel):
    """(face family, beta sign) that reproduce the body's hop term."""
    if kernel == "achimbdpsi":
        return "wilson", 1.0          # out -= beta*hop, no clover on the hops
    return {"wilson": ("wilson", -1.0), "clover": ("clover", 1.0),
            "tm": ("tm", -1.0), "tm_clover": ("tm_clover", 1.0)}[family]


class TComm:
    """Nearest-neighbour exchange along t over torch.distributed."""

    def __init__(self, group=None):
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        nccl = dist.is_initialized() and dist.get_backend(group) == "nccl"
        self.device = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")

    @property
    def fwd(self):
        return (self.rank + 1) % self.world

    @property
    def back(self):
        return (self.rank - 1) % self.world

    def start(self, send_fwd, send_back, recv_from_back, recv_from_fwd):
        """Post the four transfers; returns the request handles."""
        g = self.group
        ops = [dist.P2POp(dist.isend, send_fwd, self._peer(self.fwd), g, tag=0),
               dist.P2POp(dist.irecv, recv_from_back, self._peer(self.back), g, tag=0),
               dist.P2POp(dist.isend, send_back, self._peer(self.back), g, tag=1),
               dist.P2POp(dist.irecv, recv_from_fwd, self._peer(self.fwd), g, tag=1)]
        return dist.batch_isend_irecv(ops)

    def _peer(self, r):
        return dist.get_global_rank(self.group, r) if self.group is not None else r

    def allreduce(self, v):
        """Sum of the FP64 scalar v over the ranks."""
        if self.world == 1:
            return float(v)
        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, group=self.group)
        return float(t.item())

    @staticmethod
    def wait(reqs):
        for r in reqs:
            r.wait()


def local_geometry(g_global: Geometry, rank, world) -> Geometry:
    """The slab of `rank` of a lattice split into `world` equal t slabs."""
    if g_global.nt % world or (g_global.nt // world) % 2:
        raise ValueError("nt = %d must split into even slabs over %d ranks" % (g_global.nt, world))
    return g_global.with_(nt=g_global.nt // world, t_edge_lo=(rank == 0), t_edge_hi=(rank == world - 1))


class TSlabDslash:
    """Operator application on a t slab with halo exchange."""

    def __init__(self, g: Geometry, comm: TComm, kernels):
        self.g = g
        self.comm = comm
        self.k = kernels
        nface = g.face_sites(6)
        self.bufs = [kernels.alloc(g.face_elems * nface) for _ in range(4)]  # send fwd, send back, recv back, recv fwd

    def apply(self, family, kernel, isign, cb, psi, out, gauge, chi=None, clover=None, coeff_s=1.0,
              coeff_t_f=1.0, coeff_t_b=1.0, alpha=1.0, mu=0.0, muinv=1.0, rho=0.0, tbc_mask=0,
              tbc_phases=None):
        g = self.g
        kw = dict(chi=chi, clover=clover, coeff_s=coeff_s, coeff_t_f=coeff_t_f, coeff_t_b=coeff_t_b,
                  alpha=alpha, mu=mu, muinv=muinv, rho=rho, tbc_mask=tbc_mask, tbc_phases=tbc_phases)
        if self.comm.world == 1:
            self.k.body(g, family, kernel, isign, cb, psi, out, gauge, accumulate=None, **kw)
            return out
        send_fwd, send_back, recv_back, recv_fwd = self.bufs
        self.k.pack(g, isign, 1 - cb, psi, send_fwd, 7)
        self.k.pack(g, isign, 1 - cb, psi, send_back, 6)
        reqs = self.comm.start(send_fwd, send_back, recv_back, recv_fwd)
        self.k.body(g, family, kernel, isign, cb, psi, out, gauge, accumulate=[1, 1, 1, 1, 1, 1, 0, 0], **kw)
        self.comm.wait(reqs)
        fam, sg = face_kind(family, kernel)
        tb = g.t_boundary
        beta_b = sg * coeff_t_b * (tb if g.t_edge_lo else 1.0)
        beta_f = sg * coeff_t_f * (tb if g.t_edge_hi else 1.0)
        tbc = bool(tbc_mask & 8)
        cl = clover if fam in ("clover", "tm_clover") else None
        self.k.unpack(g, fam, isign, cb, recv_back, gauge, out, 6, beta=beta_b, clover=cl, mu=mu, muinv=muinv,
                      tbc=tbc, tbc_phases=tbc_phases)
        self.k.unpack(g, fam, isign, cb, recv_fwd, gauge, out, 7, beta=beta_f, clover=cl, mu=mu, muinv=muinv,
                      tbc=tbc, tbc_phases=tbc_phases)
        return out


class TSlabEvenOdd:
    """The even-odd operator Mhat x = A_tt x - D_to A_oo^-1 D_ot x on a t slab
    (t = target_cb, o = the other checkerboard): the plain kernel on the other
    checkerboard (hops scaled by 1/alpha for Wilson, whose A is alpha), then
    achimbdpsi on the target, each application with its halo exchange.
    gauge, clov and clov_dag are indexed by checkerboard as for
    qb200_operator (clov: A^-1 on the other checkerboard, A on the target;
    clov_dag: their adjoints, used by TM clover for Mhat^dag)."""

    def __init__(self, dslash: TSlabDslash, family, gauge, clov=(None, None), clov_dag=(None, None), target_cb=1,
                 coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0, alpha=1.0, mu=0.0, muinv=1.0, rho=0.0, tbc_mask=0,
                 tbc_phases=None):
        self.d, self.family, self.target = dslash, family, target_cb
        self.gauge, self.clov, self.clov_dag = gauge, clov, clov_dag
        self.kw = dict(coeff_s=coeff_s, coeff_t_f=coeff_t_f, coeff_t_b=coeff_t_b, alpha=alpha, mu=mu,
                       muinv=muinv, rho=rho, tbc_mask=tbc_mask, tbc_phases=tbc_phases)
        self._tmp = None

    def apply(self, x, isign=1, out=None):
        """out = Mhat x (isign +1) or Mhat^dag x (-1)."""
        k = self.d.k
        other = 1 - self.target
        out = out if out is not None else k.alloc(x.numel())
        if self._tmp is None or self._tmp.numel() != x.numel():
            self._tmp = k.alloc(x.numel())
        sc = 1.0 / self.kw["alpha"] if self.family == "wilson" else 1.0
        clov = self.clov_dag if (self.family == "tm_clover" and isign < 0) else self.clov
        k1 = dict(self.kw, coeff_s=self.kw["coeff_s"] * sc, coeff_t_f=self.kw["coeff_t_f"] * sc,
                  coeff_t_b=self.kw["coeff_t_b"] * sc)
        self.d.apply(self.family, "dslash", isign, other, x, self._tmp, self.gauge[other], clover=clov[other], **k1)
        self.d.apply(self.family, "achimbdpsi", isign, self.target, self._tmp, out, self.gauge[self.target], chi=x,
                     clover=clov[self.target], **self.kw)
        return out


def cg(op: TSlabEvenOdd, b, tol=1e-10, max_iter=10000, x=None):
    """CG on Mhat^dag Mhat x = Mhat^dag b over the t slabs (x: initial guess,
    default 0).  Every rank takes the same steps: the stopping test uses the
    all-reduced |r|^2, so the ranks leave the loop together.  Returns x and
    {"iters", "rel_res"} with rel_res = |b - Mhat x| / |b| over the whole
    lattice (FP64)."""
    k, comm = op.d.k, op.d.comm
    dot = lambda u, v: comm.allreduce(k.dot(u, v))
    x = x if x is not None else k.alloc(b.numel())
    rhs = op.apply(b, -1)
    r = op.apply(op.apply(x), -1)
    k.axpby(1.0, rhs, -1.0, r)                 # r = rhs - A x
    p = k.alloc(b.numel())
    k.axpby(1.0, r, 0.0, p)
    Ap = k.alloc(b.numel())
    t = k.alloc(b.numel())
    rr, bb = dot(r, r), dot(rhs, rhs)
    stop = tol * tol * bb
    it = 0
    while rr > stop and it < max_iter:
        op.apply(p, 1, t)
        op.apply(t, -1, Ap)
        alpha = rr / dot(p, Ap)
        k.axpby(alpha, p, 1.0, x)
        k.axpby(-alpha, Ap, 1.0, r)
        rr_new = dot(r, r)
        k.axpby(1.0, r, rr_new / rr, p)
        rr = rr_new
        it += 1
        if not math.isfinite(rr):
            raise RuntimeError("cg: residual is not finite")
    res = op.apply(x, 1, t)
    k.axpby(1.0, b, -1.0, res)                 # b - Mhat x
    rel = math.sqrt(dot(res, res) / dot(b, b))
    return x, {"iters": it, "rel_res": rel}


class GPUKernels:
    """Compute steps of TSlabDslash on the current CUDA device (FP64 BLAS of
    the slab solver through qb200_blas_axpby / qb200_blas_dot)."""

    def __init__(self, dtype, device):
        self.dtype = dtype
        self.device = device
        self._part = None
        self._res = None

    def axpby(self, a, x, b, y):
        """y = a x + b y (FP64 vectors)."""
        from . import _lib, ops
        _lib.check(_lib.lib().qb200_blas_axpby(1, x.numel(), float(a), x.data_ptr(), float(b), y.data_ptr(),
                                               ops._stream(None)))

    def dot(self, x, y):
        """Local real inner product (FP64 accumulation)."""
        from . import _lib, ops
        L = _lib.lib()
        if self._part is None:
            self._part = torch.zeros(L.qb200_blas_partials_len(), dtype=torch.float64, device=self.device)
            self._res = torch.zeros(2, dtype=torch.float64, device=self.device)
        _lib.check(L.qb200_blas_dot(1, x.numel(), x.data_ptr(), y.data_ptr(), self._res.data_ptr(),
                                    self._part.data_ptr(), ops._stream(None)))
        return float(self._res[0].item())

    def alloc(self, n):
        return torch.zeros(n, dtype=self.dtype, device=self.device)

    def body(self, g, family, kernel, isign, cb, psi, out, gauge, accumulate=None, **kw):
        from . import ops
        ops.dslash(g, family, kernel, isign, cb, psi, out, gauge, accumulate=accumulate, **kw)

    def pack(self, g, isign, psi_cb, psi, buf, dir):
        from . import ops
        ops.face_pack(g, isign, psi_cb, psi, buf, dir)

    def unpack(self, g, family, isign, cb, buf, gauge, out, dir, **kw):
        from . import ops
        ops.face_unpack(g, family, isign, cb, buf, gauge, out, dir, **kw)
