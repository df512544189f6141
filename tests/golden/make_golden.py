#!/usr/bin/env python3
"""Generate the golden vectors of tests/golden/*.npz from the reference's own
generated kernels (oracle/_ref/libqphix_ref_scalar_{f32,f64}.so, built from
the reference sources by oracle/ref_build.py).

Each file holds seeded inputs on a 4^4 lattice in the scalar QPhiX layout
(SOALEN = VECLEN = 1) and the reference's outputs for every body kernel
(4 families x {dslash, achimbdpsi} x {plus, minus} x {18, 12} links, half of
them with twisted boundary phases and some with accumulate flags cleared) and
for the face pack / unpack kernels.  tests/test_oracle_golden.py checks the
oracle against them and tests/test_golden_gpu.py the CUDA kernels.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "qphix-codegen_b200"), os.path.join(REPO, "tests")]

import helpers as H  # noqa: E402
import oracle as O  # noqa: E402
from qphix_b200.lattice import F32, F64, Geometry  # noqa: E402

DIMS = (4, 4, 4, 4)


def cases():
    i = 0
    for fam in H.FAMILIES:
        for kernel in H.KERNELS:
            for isign in (1, -1):
                for comp in (False, True):
                    tbc = 13 if i % 2 else 0
                    acc = [1, 1, 0, 1, 1, 1, 1, 0] if i % 3 == 0 else None
                    yield i, fam, kernel, isign, comp, tbc, acc
                    i += 1


def main():
    for ft, name in ((F32, "scalar_f32"), (F64, "scalar_f64")):
        if not O.ref_available(name):
            raise SystemExit("build the reference kernels first: python oracle/ref_build.py " + name)
        store = {}
        g18 = Geometry(*DIMS, soalen=1, veclen=1, ftype=ft, compress12=False, t_boundary=-1.0)
        for cb in (0, 1):
            f = H.make_fields(g18, cb=cb, seed=4242)
            for k in ("psi", "chi", "gauge", "clover", "fclover"):
                store["in_%s_cb%d" % (k, cb)] = f[k]
        for i, fam, kernel, isign, comp, tbc, acc in cases():
            cb = i % 2
            g = Geometry(*DIMS, soalen=1, veclen=1, ftype=ft, compress12=comp, t_boundary=-1.0)

            def get(k):
                a = store["in_%s_cb%d" % (k, cb)]
                if k == "gauge" and comp:
                    a = H.compress_gauge(g18, a)
                return O.aligned(a)

            pp = H.op_params(fam, kernel, tbc_mask=tbc, accumulate=acc)
            prm = O.make_params(**pp)
            cl = get("fclover" if fam == "tm_clover" else "clover")
            out = O.ref_dslash(name, g, fam, kernel, isign, cb, get("psi"), get("gauge"), chi=get("chi"),
                               clover=cl, params=prm)
            store["body_%d" % i] = out[: g.spinor_elems].copy()
            store["body_%d_meta" % i] = np.array([H.FAMILIES.index(fam), H.KERNELS.index(kernel), isign,
                                                  int(comp), tbc, -1 if acc is None else
                                                  int("".join(str(a) for a in acc), 2), cb])
        # faces: pack every dir and sign from the cb=1 psi; unpack per family
        g = Geometry(*DIMS, soalen=1, veclen=1, ftype=ft, compress12=False, t_boundary=-1.0)
        psi = O.aligned(store["in_psi_cb1"])
        for d in range(8):
            for isign in (1, -1):
                store["pack_%d_%d" % (d, isign)] = O.ref_face_pack(name, g, isign, 1, psi, d).copy()
        for fi, fam in enumerate(H.FAMILIES):
            for d in range(8):
                isign = 1 if (d + fi) % 2 else -1
                tbc = d % 3 == 0
                buf = O.aligned(store["pack_%d_%d" % (d ^ 1, isign)])
                out = O.aligned(store["in_chi_cb0"])
                cl = O.aligned(store["in_%s_cb0" % ("fclover" if fam == "tm_clover" else "clover")])
                pp = H.op_params(fam, "dslash")
                O.ref_face_unpack(name, g, fam, isign, 0, buf, O.aligned(store["in_gauge_cb0"]), out, d,
                                  beta=0.37, clover=cl, mu=pp["mu"], muinv=pp["muinv"], tbc=tbc,
                                  tbc_phases=pp["tbc_phases"])
                store["unpack_%s_%d" % (fam, d)] = out[: g.spinor_elems].copy()
                store["unpack_%s_%d_meta" % (fam, d)] = np.array([isign, int(tbc)])
        path = os.path.join(HERE, "ref_%s_4x4x4x4.npz" % name)
        np.savez_compressed(path, **store)
        print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    main()
