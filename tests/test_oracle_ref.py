"""The oracle against the reference's generated kernels run live (needs the
libraries built by oracle/ref_build.py; skipped where they are absent).
Covers the SIMD layouts (SOALEN 4/16 with VECLEN 16, AVX2 SOALEN 8, half
storage) whose x-neighbour split loads and lane masks the tile driver sets up."""
import numpy as np
import pytest

import helpers as H
import oracle as O
from qphix_b200.lattice import F16, F32, F64, Geometry

CASES = [
    ("scalar_f32", Geometry(4, 4, 4, 4, soalen=1, veclen=1, ftype=F32, t_boundary=-1.0), 1e-6),
    ("scalar_f64", Geometry(4, 4, 4, 4, soalen=1, veclen=1, ftype=F64, t_boundary=-1.0), 1e-13),
    ("avx512_f32_s4", Geometry(8, 8, 4, 4, soalen=4, veclen=16, ftype=F32, t_boundary=-1.0), 1e-6),
    ("avx512_f32_s16", Geometry(32, 4, 4, 2, soalen=16, veclen=16, ftype=F32, t_boundary=-1.0), 1e-6),
    ("avx512_f16_s4", Geometry(8, 8, 4, 4, soalen=4, veclen=16, ftype=F16, t_boundary=-1.0), 1e-3),
    ("avx2_f32_s8", Geometry(16, 4, 4, 4, soalen=8, veclen=8, ftype=F32, t_boundary=-1.0), 1e-6),
]


def _cpu_has(flag):
    try:
        return flag in open("/proc/cpuinfo").read()
    except OSError:
        return False


@pytest.mark.parametrize("name,g0,tol", CASES, ids=[c[0] for c in CASES])
def test_oracle_vs_reference(name, g0, tol):
    if not O.ref_available(name):
        pytest.skip("reference kernels %s not built" % name)
    if name.startswith("avx512") and not _cpu_has("avx512f"):
        pytest.skip("host has no AVX512")
    if name.startswith("avx2") and not _cpu_has("avx2"):
        pytest.skip("host has no AVX2")
    for comp in (False, True):
        g = g0.with_(compress12=comp)
        f = H.make_fields(g, cb=1, seed=77)
        A = {k: O.aligned(v) for k, v in f.items() if k != "U"}
        for fam in H.FAMILIES:
            for kernel in H.KERNELS:
                for isign in (1, -1):
                    for tbc, acc in ((0, None), (9, [0, 1, 1, 0, 1, 1, 0, 1])):
                        pp = H.op_params(fam, kernel, tbc_mask=tbc, accumulate=acc)
                        if g.ftype == F16:  # half kernels take binary16 scalars
                            for k in ("coeff_s", "coeff_t_f", "coeff_t_b", "alpha", "mu", "muinv", "rho"):
                                pp[k] = float(np.float16(pp[k]))
                            pp["tbc_phases"] = np.float16(np.array(pp["tbc_phases"])).astype(float).tolist()
                        prm = O.make_params(**pp)
                        cl = "fclover" if fam == "tm_clover" else "clover"
                        a = O.dslash(g, fam, kernel, isign, 1, f["psi"], f["gauge"], chi=f["chi"], clover=f[cl],
                                     params=prm)
                        b = O.ref_dslash(name, g, fam, kernel, isign, 1, A["psi"], A["gauge"], chi=A["chi"],
                                         clover=A[cl], params=prm)
                        e = H.site_rel_err(g, a, b)
                        assert e < tol, (fam, kernel, isign, comp, tbc, e)
