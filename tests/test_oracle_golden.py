"""The oracle against the reference's golden vectors (tests/golden, produced
by the reference's generated scalar kernels): every body kernel variant and
the face pack / unpack kernels."""
import numpy as np
import pytest

import helpers as H
import oracle as O
from qphix_b200.lattice import F32, F64, Geometry

TOL = {F32: 1e-6, F64: 1e-13}


def _inputs(gold, cb, comp, g18):
    def get(k):
        a = gold["in_%s_cb%d" % (k, cb)]
        if k == "gauge" and comp:
            a = H.compress_gauge(g18, a)
        return a
    return get


@pytest.mark.parametrize("ft", [F32, F64])
def test_body_kernels(ft):
    gold = H.load_golden(ft)
    g18 = Geometry(4, 4, 4, 4, soalen=1, veclen=1, ftype=ft, t_boundary=-1.0)
    n = 0
    for key in sorted(k for k in gold if k.startswith("body_") and not k.endswith("_meta")):
        fam_i, ker_i, isign, comp, tbc, acc_bits, cb = gold[key + "_meta"]
        fam, kernel = H.FAMILIES[fam_i], H.KERNELS[ker_i]
        acc = None if acc_bits < 0 else [int(c) for c in format(int(acc_bits), "08b")]
        g = g18.with_(compress12=bool(comp))
        get = _inputs(gold, cb, comp, g18)
        prm = O.make_params(**H.op_params(fam, kernel, tbc_mask=int(tbc), accumulate=acc))
        out = O.dslash(g, fam, kernel, int(isign), int(cb), get("psi"), get("gauge"), chi=get("chi"),
                       clover=get("fclover" if fam == "tm_clover" else "clover"), params=prm)
        e = H.site_rel_err(g, out, gold[key])
        assert e < TOL[ft], (key, fam, kernel, isign, comp, e)
        n += 1
    assert n == 32


@pytest.mark.parametrize("ft", [F32, F64])
def test_face_kernels(ft):
    gold = H.load_golden(ft)
    g = Geometry(4, 4, 4, 4, soalen=1, veclen=1, ftype=ft, t_boundary=-1.0)
    psi = gold["in_psi_cb1"]
    for d in range(8):
        for isign in (1, -1):
            buf = O.face_pack(g, isign, 1, psi, d)
            ref = gold["pack_%d_%d" % (d, isign)]
            assert buf.shape == ref.shape
            np.testing.assert_allclose(buf, ref, rtol=0, atol=TOL[ft] * 8)
    for fam in H.FAMILIES:
        for d in range(8):
            isign, tbc = gold["unpack_%s_%d_meta" % (fam, d)]
            pp = H.op_params(fam, "dslash")
            out = gold["in_chi_cb0"].copy()
            O.face_unpack(g, fam, int(isign), 0, gold["pack_%d_%d" % (d ^ 1, isign)], gold["in_gauge_cb0"], out,
                          d, beta=0.37, clover=gold["in_%s_cb0" % ("fclover" if fam == "tm_clover" else "clover")],
                          mu=pp["mu"], muinv=pp["muinv"], tbc=bool(tbc), tbc_phases=pp["tbc_phases"])
            e = H.site_rel_err(g, out, gold["unpack_%s_%d" % (fam, d)])
            assert e < TOL[ft], (fam, d, e)
