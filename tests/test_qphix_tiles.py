"""The per-tile QPhiX kernel interface (include/qphix_b200_qphix.h).

tests/qphix_tile_driver.cpp plays QPhiX: it is compiled against the
reference's own kernel declarations (codegen/jinja/*_decl.h.j2 rendered
unchanged into oracle/_ref/include by oracle/ref_build.py), links
libqphix_b200.so with every symbol resolved at link time, and calls the b200
specialisations tile by tile.  Checked:
  - (CPU) the link resolves every body template for every tbc combination,
    storage type and veclen = soalen of the b200 ISA, and every face
    template, by the reference's symbol names;
  - (GPU) bodies of all four families, both forms and signs, 12/18-real
    links, twisted phases and boundary masks against the reference's AVX512
    SOALEN 16 kernels on the same arrays, the FP64 oracle (helpers.TOL) and
    the lattice-level entry points (for FP32 and FP64 the same bits: both
    run the same per-site arithmetic; the lattice-level 16-bit kernel works
    on two sites per thread and may round the stored result differently);
    FP64 and half storage against the FP64 oracle;
  - (GPU) face pack and finish of every direction and family against the
    FP64 oracle, the buffers in the reference's per-tile layout
    ([2 spin][3 colour][2 re/im][lanes] per tile)."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

import helpers as H
import oracle as O
from qphix_b200 import _lib, ops
from qphix_b200.lattice import F16, F32, F64, FTYPE_NAMES, Geometry

DRIVER = os.path.join(H.REPO, "tests", "qphix_tile_driver.cpp")
DECLS = os.path.join(H.REPO, "oracle", "_ref", "include")
FAM = {"wilson": 0, "clover": 1, "tm": 2, "tm_clover": 3}
# ftype codes of the driver: 0 float, 1 double, 2 QPhiX::half
DRV_FT = {F32: 0, F64: 1, F16: 2}


def _build_driver(tmpdir):
    if not os.path.exists(os.path.join(DECLS, "dslash_decl.h")):
        pytest.fail("reference declarations missing from oracle/_ref/include (python oracle/ref_build.py)")
    if not os.path.exists(_lib.LIB_PATH):
        pytest.fail("libqphix_b200.so not built")
    libdir = os.path.dirname(_lib.LIB_PATH)
    so = os.path.join(str(tmpdir), "libqphix_tile_driver.so")
    cmd = [shutil.which("g++") or "g++", "-O1", "-std=c++14", "-fPIC", "-shared", "-w", "-I" + DECLS, DRIVER,
           "-o", so, "-L" + libdir, "-lqphix_b200", "-Wl,-rpath," + libdir, "-Wl,--no-undefined"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout[-4000:]
    L = ctypes.CDLL(so)
    I, D, P = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    L.qtd_body.argtypes = [I] * 7 + [D, I, I, I, I, I, I, I, I, I, P, P, P, P, P] + [D] * 7 + [P, P]
    L.qtd_face.argtypes = [I] * 15 + [P, P, P, P, D, D, D, P]
    L.qtd_symbols.argtypes = []
    return L


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    return _build_driver(tmp_path_factory.mktemp("qphix_tiles"))


def test_driver_links_every_b200_specialisation(driver):
    # 3 storage types x 3 veclen x 2 compressions x 16 tbc combinations,
    # 16 body templates each, all resolved by the link (--no-undefined)
    assert driver.qtd_symbols() == 288
    nm = shutil.which("nm")
    if nm:
        out = subprocess.run([nm, "-D", "--defined-only", _lib.LIB_PATH], stdout=subprocess.PIPE, text=True).stdout
        n = sum(1 for line in out.splitlines() if "_ZN5QPhiX" in line)
        # 256 body + 16 face-finish + 2 face-pack templates per (FT, veclen, compress12)
        assert n == 18 * 274, n


def _last_error():
    L = ctypes.CDLL(_lib.LIB_PATH)
    L.qb200_qphix_last_error.restype = ctypes.c_char_p
    return L.qb200_qphix_last_error()


def _ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _dptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _tile_body(L, g, fam, kernel, isign, cb, d, p, tbc, accumulate=None):
    """the body over a checkerboard through the per-tile kernels"""
    out = torch.zeros_like(d["psi"])
    ph = np.ascontiguousarray(np.asarray(p["tbc_phases"], dtype=np.float64).reshape(-1))
    acc = None if accumulate is None else np.asarray(accumulate, dtype=np.uint32)
    rc = L.qtd_body(g.nx, g.ny, g.nz, g.nt, g.soalen, g.pad_xy, g.pad_xyz, g.t_boundary, int(g.t_edge_lo),
                    int(g.t_edge_hi), DRV_FT[g.ftype], int(g.compress12), FAM[fam], int(kernel == "achimbdpsi"),
                    isign, cb, tbc, _ptr(d["psi"]), _ptr(d["chi"]), _ptr(d["gauge"]), _ptr(d["clover"]),
                    _ptr(out), p["coeff_s"], p["coeff_t_f"], p["coeff_t_b"], p["alpha"], p["mu"], p["muinv"],
                    p["rho"], _dptr(ph), _dptr(acc))
    assert rc == 0, _last_error()
    torch.cuda.synchronize()
    return out


def _fields(g, cuda, seed, cb):
    f = H.make_fields(g, cb=cb, seed=seed)
    return f, {k: H.to_torch(f[k], cuda) for k in ("psi", "chi", "gauge", "clover", "fclover")}


def _check_bodies(L, g, cuda, tbcs, ref_name=None, seed=3000):
    g64 = g.with_(ftype=F64)
    for cb in (0, 1):
        f, t = _fields(g, cuda, seed + cb, cb)
        for fam in H.FAMILIES:
            clk = "fclover" if fam == "tm_clover" else "clover"
            d = {"psi": t["psi"], "chi": t["chi"], "gauge": t["gauge"],
                 "clover": t[clk] if fam in ("clover", "tm_clover") else None}
            for kernel in H.KERNELS:
                for isign in (1, -1):
                    for tbc in tbcs:
                        acc = [1, 0, 1, 1, 0, 1, 1, 0] if tbc == tbcs[-1] else None
                        p = H.op_params(fam, kernel, seed=tbc, tbc_mask=tbc, accumulate=acc)
                        a = _tile_body(L, g, fam, kernel, isign, cb, d, p, tbc, acc)
                        # the lattice-level entry point on the same fields
                        lat = torch.zeros_like(d["psi"])
                        q = dict(p)
                        ops.dslash(g, fam, kernel, isign, cb, d["psi"], lat, d["gauge"], chi=d["chi"],
                                   clover=d["clover"], **q)
                        torch.cuda.synchronize()
                        if g.ftype in (F32, F64):
                            assert torch.equal(a, lat), (fam, kernel, isign, cb, tbc)
                        q.pop("tbc_phases")
                        q.pop("accumulate")
                        prm = O.make_params(**q, tbc_phases=p["tbc_phases"], accumulate=acc)
                        cl_np = f[clk] if fam in ("clover", "tm_clover") else None
                        b = O.dslash(g, fam, kernel, isign, cb, f["psi"], f["gauge"], chi=f["chi"], clover=cl_np,
                                     params=prm, fp64_out=True)
                        an = H.to_np(a)
                        e = H.record("per-tile %s v%d vs fp64 oracle" % (FTYPE_NAMES[g.ftype], g.veclen),
                                     H.site_rel_err(g, an, b, g64), H.TOL[g.ftype])
                        assert e < H.TOL[g.ftype], (fam, kernel, isign, cb, tbc, e)
                        if ref_name:
                            h = {k: O.aligned(v) for k, v in f.items() if k != "U"}
                            r = O.ref_dslash(ref_name, g, fam, kernel, isign, cb, h["psi"], h["gauge"], chi=h["chi"],
                                             clover=h[clk] if cl_np is not None else None, params=prm)
                            e2 = H.record("per-tile f32 v16 vs reference %s" % ref_name,
                                          H.site_rel_err(g, an, r), 2 * H.TOL[F32])
                            assert e2 < 2 * H.TOL[F32], (fam, kernel, isign, cb, tbc, e2)


@pytest.mark.gpu
def test_tile_bodies_f32_v16_vs_reference(cuda, driver):
    name = "avx512_f32_s16"
    if not O.ref_available(name):
        pytest.fail("reference kernels missing from oracle/_ref (python oracle/ref_build.py)")
    for comp in (True, False):
        g = Geometry(64, 4, 4, 4, soalen=16, veclen=16, ftype=F32, compress12=comp, t_boundary=-1.0)
        _check_bodies(driver, g, cuda, tbcs=(0, 13), ref_name=name)


@pytest.mark.gpu
@pytest.mark.parametrize("ft,v", [(F64, 4), (F16, 8), (F32, 4), (F32, 8)])
def test_tile_bodies_vs_fp64_oracle(cuda, driver, ft, v):
    g = Geometry(4 * v, 4, 4, 4, soalen=v, veclen=v, ftype=ft, compress12=(v != 8), t_boundary=-1.0)
    _check_bodies(driver, g, cuda, tbcs=(0, 11), seed=3100 + v)


def _to_tiles(g, site_major, d):
    """site-major face records (n, 12) -> the per-tile layout [12][lanes]
    of the reference (x faces: one lane per tile when veclen == soalen)"""
    a = np.asarray(site_major).reshape(-1, 12)
    if d < 2:
        return np.ascontiguousarray(a).reshape(-1)
    return np.ascontiguousarray(a.reshape(-1, g.veclen, 12).transpose(0, 2, 1)).reshape(-1)


@pytest.mark.gpu
@pytest.mark.parametrize("ft,v", [(F32, 16), (F32, 4), (F64, 8), (F16, 8)])
def test_tile_faces_vs_fp64_oracle(cuda, driver, ft, v):
    g = Geometry(4 * v, 4, 6, 4, soalen=v, veclen=v, ftype=ft, compress12=True)
    f = H.make_fields(g, cb=0, seed=3200)
    psi = H.to_torch(f["psi"], cuda)
    gauge = H.to_torch(f["gauge"], cuda)
    tol = H.TOL[ft]
    for d in range(8):
        n = g.face_sites(d)
        for isign in (1, -1):
            buf = torch.zeros(12 * n, dtype=g.dtype, device=cuda)
            rc = driver.qtd_face(g.nx, g.ny, g.nz, g.nt, v, 0, 0, DRV_FT[ft], 1, 0, isign, 1, 0, 0, d, _ptr(buf),
                                 _ptr(psi), None, None, 0.0, 0.0, 1.0, None)
            assert rc == 0, _last_error()
            torch.cuda.synchronize()
            ref = O.face_pack(g, isign, 1, f["psi"], d, fp64_out=True)
            got = buf.cpu().double().numpy()
            e = H.record("per-tile face pack %s v%d" % (FTYPE_NAMES[ft], v),
                         H.face_rel_err(got, _to_tiles(g, ref, d)), tol)
            assert e < tol, (d, isign, e)
    for fam in H.FAMILIES:
        cl_np = f["fclover" if fam == "tm_clover" else "clover"]
        cl = H.to_torch(cl_np, cuda)
        for d in range(8):
            for isign in (1, -1):
                src = H.make_fields(g, cb=1, seed=3300 + d)["psi"]
                inbuf_np = O.face_pack(g, isign, 1, src, d ^ 1)
                pp = H.op_params(fam, "dslash")
                tbc = (d + isign) % 3 == 0
                ph = np.ascontiguousarray(np.asarray(pp["tbc_phases"], dtype=np.float64).reshape(-1))
                out = H.to_torch(f["chi"], cuda)
                inbuf = H.to_torch(_to_tiles(g, inbuf_np, d), cuda)
                rc = driver.qtd_face(g.nx, g.ny, g.nz, g.nt, v, 0, 0, DRV_FT[ft], 1, FAM[fam], isign, 0, 1,
                                     int(tbc), d, _ptr(inbuf), _ptr(out), _ptr(gauge), _ptr(cl), 0.41, pp["mu"],
                                     pp["muinv"], _dptr(ph))
                assert rc == 0, _last_error()
                torch.cuda.synchronize()
                ref = O.face_unpack(g, fam, isign, 0, inbuf_np, f["gauge"], H.as_f64(g, f["chi"]), d, beta=0.41,
                                    clover=cl_np, mu=pp["mu"], muinv=pp["muinv"], tbc=tbc,
                                    tbc_phases=pp["tbc_phases"], fp64_out=True)
                e = H.record("per-tile face finish %s v%d" % (FTYPE_NAMES[ft], v),
                             H.site_rel_err(g, H.to_np(out), ref, g.with_(ftype=F64)), tol)
                assert e < tol, (fam, d, isign, e)
