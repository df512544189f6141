"""Backward pass of the hopping term: link force kernels and autograd bindings.

The reference (qphix-codegen) generates forward kernels only; this module
adds the derivatives a gauge-field update needs, built on qb200_hop_force
(include/qphix_b200.h) and the forward kernels:

  * `hop_force`: for L = Re <chi, H_cb psi> (H_cb the plain Wilson hopping
    term on checkerboard cb, codegen/dslash_common.cc:1729-1826), the
    derivative dL/dU of every stored link of cb, or its su(3) projection
    TA(dL/dU U^dag);
  * `links_grad`: the per-checkerboard derivatives folded onto the
    full-lattice links U[mu][t][z][y][x] (each link is stored twice: as the
    forward link of x and the backward link of x + mu);
  * `WilsonHop` (torch.autograd.Function): out = H_cb(U) psi with gradients
    for psi (the dagger dslash, isign flipped, on the other checkerboard) and
    for U (the force kernel);
  * `PseudofermionAction`: S = phi^dag (Mhat^dag Mhat)^-1 phi for the
    even-odd Schur operator of any family, with dS/dU from two force
    launches and dS/dphi = 2 (Mhat^dag Mhat)^-1 phi.

Complex gradients follow torch's convention for a real loss:
dL/dRe z + i dL/dIm z.  The clover field is an independent input (its own
dependence on U is not part of the operator family), and the lattice is a
single local volume (t_edge_lo = t_edge_hi = True).
"""
import ctypes

import torch

from . import _lib, layout, ops
from .lattice import F32, F64, Geometry

_INDEX_CACHE = {}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _nsites(g: Geometry):
    return g.nxh * g.ny * g.nz * g.nt


def hop_force(g: Geometry, cb, isign, chi, psi, gauge=None, *, coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0,
              tbc_mask=0, tbc_phases=None, out=None):
    """qb200_hop_force: (144 * sites of cb) reals in the storage dtype,
    component k = ((dir*3 + row)*3 + col)*2 + re/im of site i at [k*n + i]."""
    if g.ftype not in (F32, F64):
        raise ValueError("the force kernel supports FP32 and FP64 storage")
    n = 144 * _nsites(g)
    out = out if out is not None else torch.empty(n, dtype=g.dtype, device=psi.device)
    ops._check_field("chi", chi, g, g.spinor_elems)
    ops._check_field("psi", psi, g, g.spinor_elems)
    ops._check_field("force", out, g, n)
    if gauge is not None:
        ops._check_field("gauge", gauge, g, g.gauge_elems)
    lat = g.c_struct()
    P = ops._ptr
    _lib.check(_lib.lib().qb200_hop_force(ctypes.byref(lat), cb, isign, P(chi), P(psi), P(gauge), coeff_s,
                                          coeff_t_f, coeff_t_b, ctypes.c_uint(int(tbc_mask)),
                                          _lib.phases(tbc_phases), P(out), _stream()))
    return out


def force_sites(g: Geometry, force):
    """Kernel output -> complex (nt, nz, ny, nxh, 8, 3, 3)."""
    v = force.view(8, 3, 3, 2, g.nt, g.nz, g.ny, g.nxh).permute(4, 5, 6, 7, 0, 1, 2, 3).contiguous()
    return torch.view_as_complex(v)


def link_index(g: Geometry, cb, device):
    """Flat index into U.view(4 * nt*nz*ny*nx, 3, 3) of the link each stored
    slot of checkerboard cb holds, shape (nt, nz, ny, nxh, 8)."""
    key = (g.dims, cb, str(device))
    if key not in _INDEX_CACHE:
        x, y, z, t = layout.cb_coords(g, cb, device)
        L = [g.nx, g.ny, g.nz, g.nt]
        vol = g.nx * g.ny * g.nz * g.nt
        idx = []
        for mu in range(4):
            c = [x, y, z, t]
            cm = list(c)
            cm[mu] = (c[mu] - 1) % L[mu]
            lin = lambda q: ((q[3] * g.nz + q[2]) * g.ny + q[1]) * g.nx + q[0]  # noqa: E731
            idx += [mu * vol + lin(cm), mu * vol + lin(c)]
        _INDEX_CACHE[key] = torch.stack(idx, dim=4).contiguous()
    return _INDEX_CACHE[key]


def links_grad(g: Geometry, cb, force, out=None, dtype=torch.complex128):
    """Fold the force of checkerboard cb onto full-lattice links: returns (or
    accumulates into) a complex (4, nt, nz, ny, nx, 3, 3) tensor."""
    F = force_sites(g, force).to(dtype)
    vol = g.nx * g.ny * g.nz * g.nt
    if out is None:
        out = torch.zeros((4, g.nt, g.nz, g.ny, g.nx, 3, 3), dtype=dtype, device=force.device)
    idx = link_index(g, cb, force.device).reshape(-1)
    out.view(4 * vol, 3, 3).index_add_(0, idx, F.reshape(-1, 3, 3))
    return out


def su3_project(M):
    """Traceless anti-Hermitian part TA(M) = (M - M^dag)/2 - tr(M - M^dag)/6."""
    A = 0.5 * (M - M.conj().transpose(-1, -2))
    tr = torch.diagonal(A, dim1=-2, dim2=-1).sum(-1) / 3.0
    return A - tr[..., None, None] * torch.eye(3, dtype=M.dtype, device=M.device)


def link_force(U, grad_U):
    """su(3) force of a link gradient: TA(grad_U U^dag); dL/deps along
    U -> exp(eps X) U is sum Re tr(X^dag P)."""
    return su3_project(grad_U @ U.conj().transpose(-1, -2))


def _check_geometry(g: Geometry):
    if g.compress12:
        raise ValueError("the differentiable operator packs 18-real links (compress12=False)")
    if g.ftype not in (F32, F64):
        raise ValueError("the differentiable operator supports FP32 and FP64 storage")
    if not (g.t_edge_lo and g.t_edge_hi):
        raise ValueError("the differentiable operator covers a whole lattice (one t slab)")


class WilsonHop(torch.autograd.Function):
    """out = H_cb(U) psi: the plain Wilson dslash (qb200_dslash_plus_vec /
    _minus_vec) on checkerboard cb, psi on 1 - cb in the packed spinor layout,
    U the full-lattice links (complex).

        out = WilsonHop.apply(psi, U, g, cb, isign, coeffs)

    coeffs: dict with any of coeff_s, coeff_t_f, coeff_t_b, tbc_mask, tbc_phases.
    """

    @staticmethod
    def forward(ctx, psi, U, g, cb, isign, coeffs=None):
        _check_geometry(g)
        kw = dict(coeffs or {})
        gauge = layout.pack_gauge(g, U.detach(), cb)
        out = torch.zeros(g.spinor_elems, dtype=g.dtype, device=psi.device)
        ops.dslash(g, "wilson", "dslash", isign, cb, psi.detach().contiguous(), out, gauge, **kw)
        ctx.save_for_backward(psi, U)
        ctx.g, ctx.cb, ctx.isign, ctx.kw = g, cb, isign, kw
        return out

    @staticmethod
    def backward(ctx, gout):
        psi, U = ctx.saved_tensors
        g, cb, isign, kw = ctx.g, ctx.cb, ctx.isign, ctx.kw
        gout = gout.contiguous().to(g.dtype)
        gpsi = gU = None
        if ctx.needs_input_grad[0]:
            # H_cb(isign)^dag = H_{1-cb}(-isign) with the time coefficients
            # exchanged (a forward hop's adjoint is the neighbour's backward hop)
            dkw = dict(kw)
            dkw["coeff_t_f"], dkw["coeff_t_b"] = kw.get("coeff_t_b", 1.0), kw.get("coeff_t_f", 1.0)
            gauge_o = layout.pack_gauge(g, U.detach(), 1 - cb)
            gpsi = torch.zeros_like(psi)
            ops.dslash(g, "wilson", "dslash", -isign, 1 - cb, gout, gpsi, gauge_o, **dkw)
        if ctx.needs_input_grad[1]:
            F = hop_force(g, cb, isign, gout, psi.detach().contiguous(), **kw)
            gU = links_grad(g, cb, F, dtype=U.dtype)
        return gpsi, gU, None, None, None, None


def _first_step(g, family, op_kw, isign, oc, inp, gauge, clov, clov_dag):
    """The other-checkerboard half of the Schur operator (qb200_schur_apply's
    first launch): A_ee^-1 D_eo^(isign) inp."""
    out = torch.zeros(g.spinor_elems, dtype=g.dtype, device=inp.device)
    kw = dict(coeff_s=op_kw["coeff_s"], coeff_t_f=op_kw["coeff_t_f"], coeff_t_b=op_kw["coeff_t_b"],
              tbc_mask=op_kw["tbc_mask"], tbc_phases=op_kw["tbc_phases"])
    if family == "wilson":
        a = op_kw["alpha"]
        kw.update(coeff_s=kw["coeff_s"] / a, coeff_t_f=kw["coeff_t_f"] / a, coeff_t_b=kw["coeff_t_b"] / a)
    elif family == "tm":
        kw.update(mu=op_kw["mu"], muinv=op_kw["muinv"])
    elif family == "clover":
        kw.update(clover=clov[oc])
    else:
        kw.update(clover=clov[oc] if isign > 0 else clov_dag[oc])
    ops.dslash(g, family, "dslash", isign, oc, inp, out, gauge[oc], **kw)
    return out


class PseudofermionAction(torch.autograd.Function):
    """S = phi^dag (Mhat^dag Mhat)^-1 phi, Mhat the even-odd Schur operator of
    qb200_schur_apply on target_cb, solved by CG on the GPU (FP64 storage).

        S = PseudofermionAction.apply(U, phi, g, family, op_kw, clov, clov_dag, tol)

    op_kw: dict of coeff_s, coeff_t_f, coeff_t_b, alpha, mu, muinv, rho,
    tbc_mask, tbc_phases, target_cb.  clov / clov_dag: per-checkerboard packed
    fields as for EvenOddOperator (A^-1 on the other checkerboard, A on the
    target one), treated as constants.

    dS = -2 Re <Y, dMhat X> with X = (Mhat^dag Mhat)^-1 phi, Y = Mhat X and
    dMhat = -dD_oe A^-1 D_eo - D_oe A^-1 dD_eo, so
    dS/dU = 2 F_o(Y, A^-1 D_eo X) + 2 F_e(A^-dag D_eo^dag Y, X),
    F_cb(chi, psi) the hop force of checkerboard cb.
    """

    @staticmethod
    def forward(ctx, U, phi, g, family, op_kw, clov=(None, None), clov_dag=(None, None), tol=1e-12):
        from .solver import EvenOddOperator
        _check_geometry(g)
        if g.ftype != F64:
            raise ValueError("the pseudofermion action is solved in FP64 storage")
        kw = dict(coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0, alpha=1.0, mu=0.0, muinv=1.0, rho=0.0, tbc_mask=0,
                  tbc_phases=None, target_cb=1)
        kw.update(op_kw or {})
        if kw["coeff_t_f"] != kw["coeff_t_b"]:
            raise ValueError("the Schur dagger needs coeff_t_f == coeff_t_b")
        Ud = U.detach()
        gauge = (layout.pack_gauge(g, Ud, 0), layout.pack_gauge(g, Ud, 1))
        op = EvenOddOperator(g, family, gauge, clov=clov, clov_dag=clov_dag, **kw)
        X, info = op.cg_normal(phi.detach().contiguous(), tol=tol, max_iter=20000)
        ctx.save_for_backward(U, phi, X)
        ctx.g, ctx.family, ctx.kw, ctx.clov, ctx.clov_dag, ctx.op = g, family, kw, clov, clov_dag, op
        ctx.gauge = gauge
        ctx.info = info
        return (phi.detach().to(torch.float64) * X).sum()

    @staticmethod
    def backward(ctx, gS):
        U, phi, X = ctx.saved_tensors
        g, family, kw = ctx.g, ctx.family, ctx.kw
        gU = gphi = None
        if ctx.needs_input_grad[0]:
            tc = kw["target_cb"]
            oc = 1 - tc
            Y = ctx.op.apply(X, isign=1)
            Z = _first_step(g, family, kw, 1, oc, X, ctx.gauge, ctx.clov, ctx.clov_dag)
            W = _first_step(g, family, kw, -1, oc, Y, ctx.gauge, ctx.clov, ctx.clov_dag)
            fk = dict(coeff_s=kw["coeff_s"], coeff_t_f=kw["coeff_t_f"], coeff_t_b=kw["coeff_t_b"],
                      tbc_mask=kw["tbc_mask"], tbc_phases=kw["tbc_phases"])
            gU = links_grad(g, tc, hop_force(g, tc, 1, Y, Z, **fk), dtype=U.dtype)
            links_grad(g, oc, hop_force(g, oc, 1, W, X, **fk), out=gU, dtype=U.dtype)
            gU = gU * (2.0 * gS)
        if ctx.needs_input_grad[1]:
            gphi = (2.0 * gS) * X
        return gU, gphi, None, None, None, None, None, None
