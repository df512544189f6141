"""Domain decomposition of the dslash over a z x t grid of ranks (one GPU
per rank): t slabs first, then z (pz x pt ranks; pz = 1 gives plain t
slabs).

Rank r sits at grid coordinates (rz, rt) = (r % pz, r // pz) and holds the
local lattice of nz = NZ/pz slices in z and nt = NT/pt slices in t starting
at z0 = rz*nz, t0 = rt*nt (both even, so local and global checkerboards
agree).  One application of an operator on checkerboard cb is, for every
split dimension mu (z: dirs 4, 5; t: dirs 6, 7):

  1. face_proj_dir (dirs 2mu+1 and 2mu): project the sites of psi on the
     forward / backward face for the neighbour beyond it
     (codegen/dslash.cc:433-458);
  2. exchange the face buffers with the two neighbours along mu;
  3. body kernel with accumulate[2mu] = accumulate[2mu+1] = 0 for every split
     mu: every hop except the ones that leave the local block (this overlaps
     step 2);
  4. face_*finish_dir (dirs 2mu and 2mu+1): add the received faces
     (codegen/dslash.cc:463-553).

The dslash couples nearest neighbours only, so no edge or corner exchange is
needed.  The face kernels of the reference subtract beta*hop for Wilson and
twisted mass and add beta*A*hop for clover / TM clover
(dslash_common.cc:1975-1981), so each (family, kernel) pair maps to one face
kind and a sign of beta (see `face_kind`).  The beta of a z face is coeff_s;
a t face gets coeff_t_b / coeff_t_f, times the time-boundary factor on the
faces that cross the global t edge (grid row rt = 0 backward, rt = pt-1
forward).

The compute steps are delegated to a `kernels` object (GPU kernels through
the C-ABI, or the CPU oracle in the tests) and the exchange to `GridComm`, so
the same orchestration runs over NCCL on GPUs and over gloo on CPU.

`TSlabEvenOdd` composes two such applications into the even-odd operator
Mhat (the composition of qb200_schur_apply), and `cg` solves Mhat^dag Mhat
x = Mhat^dag b over the blocks: vectors stay local, each inner product is a
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


class GridComm:
    """Nearest-neighbour exchange on a pz x pt grid of ranks over
    torch.distributed (rank = rt * pz + rz).  pz = None: every rank in t."""

    def __init__(self, pz=None, group=None):
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.pz = 1 if pz is None else int(pz)
        if self.pz < 1 or self.world % self.pz:
            raise ValueError("pz = %d does not divide the %d ranks" % (self.pz, self.world))
        self.pt = self.world // self.pz
        self.rz, self.rt = self.rank % self.pz, self.rank // self.pz
        nccl = dist.is_initialized() and dist.get_backend(group) == "nccl"
        self.device = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")

    def parts(self, mu):
        """ranks along dimension mu (2 = z, 3 = t; x and y are never split)"""
        return {2: self.pz, 3: self.pt}.get(mu, 1)

    def neighbour(self, mu, step):
        rz, rt = self.rz, self.rt
        if mu == 2:
            rz = (rz + step) % self.pz
        else:
            rt = (rt + step) % self.pt
        return rt * self.pz + rz

    def start(self, mu, send_fwd, send_back, recv_from_back, recv_from_fwd):
        """Post the four transfers along mu; returns the request handles.
        With two ranks along mu both neighbours are the same rank: the two
        messages each way are told apart by tag (gloo) and by order (NCCL)."""
        g, fwd, back = self.group, self.neighbour(mu, 1), self.neighbour(mu, -1)
        ops = [dist.P2POp(dist.isend, send_fwd, self._peer(fwd), g, tag=2 * mu),
               dist.P2POp(dist.irecv, recv_from_back, self._peer(back), g, tag=2 * mu),
               dist.P2POp(dist.isend, send_back, self._peer(back), g, tag=2 * mu + 1),
               dist.P2POp(dist.irecv, recv_from_fwd, self._peer(fwd), g, tag=2 * mu + 1)]
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


class TComm(GridComm):
    """Every rank along t (pz = 1): the t-slab decomposition."""

    def __init__(self, group=None):
        super().__init__(1, group)

    @property
    def fwd(self):
        return self.neighbour(3, 1)

    @property
    def back(self):
        return self.neighbour(3, -1)


def grid_geometry(g_global: Geometry, rank, pz, pt) -> Geometry:
    """The block of `rank` (rz = rank % pz, rt = rank // pz) of a lattice
    split into pz x pt equal blocks in z and t."""
    if g_global.nz % pz or (g_global.nz // pz) % 2:
        raise ValueError("nz = %d must split into even blocks over %d ranks" % (g_global.nz, pz))
    if g_global.nt % pt or (g_global.nt // pt) % 2:
        raise ValueError("nt = %d must split into even slabs over %d ranks" % (g_global.nt, pt))
    rt = rank // pz
    return g_global.with_(nz=g_global.nz // pz, nt=g_global.nt // pt, t_edge_lo=(rt == 0),
                          t_edge_hi=(rt == pt - 1))


def local_geometry(g_global: Geometry, rank, world) -> Geometry:
    """The slab of `rank` of a lattice split into `world` equal t slabs."""
    return grid_geometry(g_global, rank, 1, world)


class HaloDslash:
    """Operator application on a z x t block with halo exchange."""

    def __init__(self, g: Geometry, comm: GridComm, kernels):
        self.g = g
        self.comm = comm
        self.k = kernels
        self.split = [mu for mu in (2, 3) if comm.parts(mu) > 1]
        # per split mu: send fwd, send back, recv from back, recv from fwd
        self.bufs = {mu: [kernels.alloc(g.face_elems * g.face_sites(2 * mu)) for _ in range(4)]
                     for mu in self.split}

    def apply(self, family, kernel, isign, cb, psi, out, gauge, chi=None, clover=None, coeff_s=1.0,
              coeff_t_f=1.0, coeff_t_b=1.0, alpha=1.0, mu=0.0, muinv=1.0, rho=0.0, tbc_mask=0,
              tbc_phases=None):
        g = self.g
        kw = dict(chi=chi, clover=clover, coeff_s=coeff_s, coeff_t_f=coeff_t_f, coeff_t_b=coeff_t_b,
                  alpha=alpha, mu=mu, muinv=muinv, rho=rho, tbc_mask=tbc_mask, tbc_phases=tbc_phases)
        if not self.split:
            self.k.body(g, family, kernel, isign, cb, psi, out, gauge, accumulate=None, **kw)
            return out
        reqs = []
        acc = [1] * 8
        for d in self.split:
            send_fwd, send_back, recv_back, recv_fwd = self.bufs[d]
            self.k.pack(g, isign, 1 - cb, psi, send_fwd, 2 * d + 1)
            self.k.pack(g, isign, 1 - cb, psi, send_back, 2 * d)
            reqs += self.comm.start(d, send_fwd, send_back, recv_back, recv_fwd)
            acc[2 * d] = acc[2 * d + 1] = 0
        self.k.body(g, family, kernel, isign, cb, psi, out, gauge, accumulate=acc, **kw)
        self.comm.wait(reqs)
        fam, sg = face_kind(family, kernel)
        tb = g.t_boundary
        cl = clover if fam in ("clover", "tm_clover") else None
        for d in self.split:
            _, _, recv_back, recv_fwd = self.bufs[d]
            if d == 3:
                beta_b = sg * coeff_t_b * (tb if g.t_edge_lo else 1.0)
                beta_f = sg * coeff_t_f * (tb if g.t_edge_hi else 1.0)
            else:
                beta_b = beta_f = sg * coeff_s
            tbc = bool(tbc_mask & (1 << d))
            self.k.unpack(g, fam, isign, cb, recv_back, gauge, out, 2 * d, beta=beta_b, clover=cl, mu=mu,
                          muinv=muinv, tbc=tbc, tbc_phases=tbc_phases)
            self.k.unpack(g, fam, isign, cb, recv_fwd, gauge, out, 2 * d + 1, beta=beta_f, clover=cl, mu=mu,
                          muinv=muinv, tbc=tbc, tbc_phases=tbc_phases)
        return out


# the t-slab form (a GridComm with pz = 1 splits t only)
TSlabDslash = HaloDslash


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
