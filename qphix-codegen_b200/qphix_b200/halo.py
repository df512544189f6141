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
"""
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


class GPUKernels:
    """Compute steps of TSlabDslash on the current CUDA device."""

    def __init__(self, dtype, device):
        self.dtype = dtype
        self.device = device

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
