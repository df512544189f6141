"""The CUDA kernels against the reference's golden vectors (tests/golden:
outputs of the reference's own scalar kernels), scalar layout, FP32 and FP64,
through the C-ABI.  Tolerances helpers.TOL (FP32 1e-6, FP64 1e-13)."""
import numpy as np
import pytest
import torch

import helpers as H
from qphix_b200 import ops
from qphix_b200.lattice import F32, F64, Geometry

pytestmark = pytest.mark.gpu
TOL = H.TOL


@pytest.mark.parametrize("ft", [F32, F64])
def test_body_kernels_vs_reference_vectors(cuda, ft):
    gold = H.load_golden(ft)
    g18 = Geometry(4, 4, 4, 4, soalen=1, veclen=1, ftype=ft, t_boundary=-1.0)
    n = 0
    for key in sorted(k for k in gold if k.startswith("body_") and not k.endswith("_meta")):
        fam_i, ker_i, isign, comp, tbc, acc_bits, cb = (int(v) for v in gold[key + "_meta"])
        fam, kernel = H.FAMILIES[fam_i], H.KERNELS[ker_i]
        acc = None if acc_bits < 0 else [int(c) for c in format(acc_bits, "08b")]
        g = g18.with_(compress12=bool(comp))
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
        gauge = gold["in_gauge_cb%d" % cb]
        if comp:
            gauge = H.compress_gauge(g18, gauge)
        psi = T(gold["in_psi_cb%d" % cb])
        out = torch.zeros_like(psi)
        pp = H.op_params(fam, kernel, tbc_mask=tbc, accumulate=acc)
        ops.dslash(g, fam, kernel, isign, cb, psi, out, T(gauge), chi=T(gold["in_chi_cb%d" % cb]),
                   clover=T(gold["in_%s_cb%d" % ("fclover" if fam == "tm_clover" else "clover", cb)]), **pp)
        e = H.site_rel_err(g, out.cpu().numpy(), gold[key])
        H.record("golden body %s" % ("f64" if ft == F64 else "f32"), e, TOL[ft])
        assert e < TOL[ft], (key, fam, kernel, isign, comp, e)
        n += 1
    assert n == 32


@pytest.mark.parametrize("ft", [F32, F64])
def test_face_kernels_vs_reference_vectors(cuda, ft):
    gold = H.load_golden(ft)
    g = Geometry(4, 4, 4, 4, soalen=1, veclen=1, ftype=ft, t_boundary=-1.0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    psi = T(gold["in_psi_cb1"])
    for d in range(8):
        for isign in (1, -1):
            ref = gold["pack_%d_%d" % (d, isign)]
            buf = torch.zeros(ref.size, dtype=g.dtype, device=cuda)
            ops.face_pack(g, isign, 1, psi, buf, d)
            e = H.record("golden face pack %s" % ("f64" if ft == F64 else "f32"),
                         H.face_rel_err(buf.cpu().numpy(), ref), TOL[ft])
            assert e < TOL[ft], (d, isign, e)
    for fam in H.FAMILIES:
        for d in range(8):
            isign, tbc = (int(v) for v in gold["unpack_%s_%d_meta" % (fam, d)])
            pp = H.op_params(fam, "dslash")
            out = T(gold["in_chi_cb0"])
            ops.face_unpack(g, fam, isign, 0, T(gold["pack_%d_%d" % (d ^ 1, isign)]), T(gold["in_gauge_cb0"]), out,
                            d, beta=0.37, clover=T(gold["in_%s_cb0" % ("fclover" if fam == "tm_clover" else "clover")]),
                            mu=pp["mu"], muinv=pp["muinv"], tbc=bool(tbc), tbc_phases=pp["tbc_phases"])
            e = H.site_rel_err(g, out.cpu().numpy(), gold["unpack_%s_%d" % (fam, d)])
            H.record("golden face unpack %s" % ("f64" if ft == F64 else "f32"), e, TOL[ft])
            assert e < TOL[ft], (fam, d, e)
