#!/usr/bin/env python3
"""Build the reference's own dslash kernels into oracle/_ref (TEST INFRASTRUCTURE).

Recipe, per configuration (ISA, precision, SOALEN, low precision):
  1. compile the reference's code generator straight from its sources in
     codegen/*.cc with g++ and the define set that the reference's
     CMakeLists.txt:151-239 uses for that ISA (setup_defs, :11-120); the one
     configured header it needs, output_dir.h (template codegen/output_dir.h.in),
     is written here;
  2. run the generator: it writes the straight-line kernel bodies
     (codegen/dslash.cc:568-751) under oracle/_ref/<cfg>/generated/;
  3. write wrapper translation units (this script's own code) that place each
     generated body inside a function whose locals carry the argument names of
     the kernel signatures (codegen/jinja/*_decl.h.j2) and register it in the
     tables of oracle/ref_driver.h;
  4. compile wrappers + oracle/ref_driver.cpp into
     oracle/_ref/libqphix_ref_<cfg>.so.
The reference's CMake/Jinja library build (generate_files.py, the generated
CMake project) is not used.  Nothing of the reference checkout is copied into the
repository: generated sources and binaries stay in the git-ignored
oracle/_ref/.  A machine without the reference sources uses the prebuilt .so.

The reference checkout is taken from --ref DIR, else from the environment
variable QPHIX_CODEGEN_REF, else from the mount point this recipe was written
for (DEFAULT_REF); DIR is the checkout's root (it holds codegen/).

Usage: python oracle/ref_build.py [--ref DIR] [cfg ...]   (default: the DEFAULT list)
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
DEFAULT_REF = "/root/reference"
REF = None  # codegen/ of the reference checkout, set by set_reference()


def reference_dir(explicit=None):
    """The reference checkout's root, or None when its sources are absent."""
    root = explicit or os.environ.get("QPHIX_CODEGEN_REF") or DEFAULT_REF
    return root if os.path.isdir(os.path.join(root, "codegen")) else None


def set_reference(root):
    global REF
    REF = os.path.join(root, "codegen")
OUT = os.path.join(HERE, "_ref")

# CMakeLists.txt:151-239 define sets (PREF_* and USE_SHUFFLES off everywhere)
COMMON = ["SERIAL_SPIN", "USE_LDUNPK", "USE_PKST", "ENABLE_STREAMING_STORES",
          "USE_PACKED_GAUGES", "USE_PACKED_CLOVER"]
ISA_DEFS = {
    "scalar": COMMON + ["NO_HW_MASKING", "NO_MASKS"],
    "avx2": COMMON + ["NO_HW_MASKING", "AVX2"],
    "avx512": COMMON + ["AVX512"],
}
ISA_CFLAGS = {
    "scalar": [],
    "avx2": ["-mavx2", "-mfma", "-mf16c"],
    "avx512": ["-mavx512f", "-mf16c", "-mfma"],
}
VECLEN = {("scalar", 1): 1, ("scalar", 2): 1, ("avx2", 1): 8, ("avx2", 2): 4,
          ("avx512", 1): 16, ("avx512", 2): 8}

# name -> (isa, precision, soalen, lowprec)
CONFIGS = {
    "scalar_f32": ("scalar", 1, 1, False),
    "scalar_f64": ("scalar", 2, 1, False),
    "avx512_f32_s4": ("avx512", 1, 4, False),
    "avx512_f32_s8": ("avx512", 1, 8, False),
    "avx512_f32_s16": ("avx512", 1, 16, False),
    "avx512_f64_s4": ("avx512", 2, 4, False),
    "avx512_f16_s4": ("avx512", 1, 4, True),
    "avx512_f16_s16": ("avx512", 1, 16, True),
    "avx2_f32_s4": ("avx2", 1, 4, False),
    "avx2_f32_s8": ("avx2", 1, 8, False),
}
DEFAULT = ["scalar_f32", "scalar_f64", "avx512_f32_s4", "avx512_f32_s16",
           "avx512_f16_s4", "avx2_f32_s8"]

FAMILIES = [  # (tm prefix, clover)
    ("", False), ("", True), ("tm_", False), ("tm_", True)]
DIRNAME = ["back", "forw"]
DIMCHAR = "XYZT"


def sh(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True)
    if r.returncode:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout[-4000:]))
    return r.stdout


def type_names(prec, lowprec):
    if lowprec:
        return "half"
    return "float" if prec == 1 else "double"


def body_file(fam, kernel, plus, comp12, tbc, tn, V, S):
    tm, clov = FAMILIES[fam]
    cp = ("clov_%s_" % tn) if clov else ""
    letters = "".join("t" if (tbc >> mu) & 1 else "s" for mu in range(4))
    return "%s%s%s_%s_body_%s_%s_v%d_s%d_%d_%s" % (
        tm, cp, kernel, "plus" if plus else "minus", tn, tn, V, S,
        12 if comp12 else 18, letters)


def unpack_file(fam, d, plus, comp12, tbc, tn, V, S):
    tm, clov = FAMILIES[fam]
    cp = ("clov_%s_" % tn) if clov else ""
    return "%s%sdslash_face_unpack_from_%s_%s_%s_%s_%s_v%d_s%d_%d_%s" % (
        tm, cp, DIRNAME[d % 2], DIMCHAR[d // 2], "plus" if plus else "minus",
        tn, tn, V, S, 12 if comp12 else 18, "t" if tbc else "s")


def pack_file(d, plus, tn, V, S):
    return "dslash_face_pack_to_%s_%s_%s_%s_%s_v%d_s%d" % (
        DIRNAME[d % 2], DIMCHAR[d // 2], "plus" if plus else "minus", tn, tn, V, S)


PROLOGUE = """\
  typedef QPhiX::Types<FT, RD_VEC, RD_SOA, {comp}> T;
  const T::FourSpinorBlock *xyBase = A.xyBase, *zbBase = A.zbBase,
      *zfBase = A.zfBase, *tbBase = A.tbBase, *tfBase = A.tfBase,
      *chiBase = A.chiBase;
  T::FourSpinorBlock *oBase = A.oBase;
  const T::SU3MatrixBlock *gBase = (const T::SU3MatrixBlock *)A.gBase;
  const T::{cltype} *clBase = (const T::{cltype} *)A.clBase;
  const int *xbOffs = A.xbOffs, *xfOffs = A.xfOffs, *ybOffs = A.ybOffs,
      *yfOffs = A.yfOffs, *offs = A.offs, *gOffs = A.gOffs;
  const unsigned int *accumulate = A.accumulate;
  const FT coeff_s = A.coeff_s, coeff_t_f = A.coeff_t_f, coeff_t_b = A.coeff_t_b,
      alpha = A.alpha, mu = A.mu, muinv = A.muinv,
      prec_mass_rho = A.prec_mass_rho, beta = A.beta;
  const FT(*tbc_phases)[2] = A.tbc_phases;
  FT *outbuf = A.outbuf;
  const FT *inbuf = A.inbuf;
  unsigned int mask = A.mask;
  int dir = A.dir;
  const int siprefdist1 = 0, siprefdist2 = 0, siprefdist3 = 0, siprefdist4 = 0,
      gprefdist = 0, clprefdist = 0, chiprefdist = 0, hsprefdist = 0,
      soprefdist = 0, si_prefdist = 0;
  const int *pfyOffs = A.offs;
  const T::FourSpinorBlock *pfBase2 = A.xyBase, *pfBase3 = A.xyBase,
      *pfBase4 = A.xyBase, *pfBaseChi = A.xyBase;
"""


def _wrap_fn(lines, fn, path, comp, cltype):
    if not os.path.exists(path):
        raise RuntimeError("missing generated kernel " + path)
    lines.append("static void %s(const TileArgs &A) {" % fn)
    lines.append(PROLOGUE.format(comp="true" if comp else "false", cltype=cltype))
    lines.append('#include "%s"' % path)
    lines.append("}")


def write_wrappers(cfgdir, gendir, tn, V, S):
    """One translation unit per (family, kernel) body set, one per family of
    face unpack kernels and one for the face pack kernels, so that g++ can
    compile them in parallel."""
    files = []

    def emit(fname, fill, lines, regs):
        lines.append("void %s() {" % fill)
        lines += regs
        lines.append("}")
        p = os.path.join(cfgdir, fname)
        open(p, "w").write("\n".join(lines) + "\n")
        files.append(p)

    glue = ['#include "ref_driver.h"', ""]
    for fam in range(4):
        cltype = "FullCloverBlock" if fam == 3 else "CloverBlock"
        parts = []
        for ach, kernel in enumerate(["dslash", "dslash_achimbdpsi"]):
            lines, regs = ['#include "ref_driver.h"', ""], []
            for plus in (0, 1):
                for comp in (0, 1):
                    for tbc in range(16):
                        fn = "b_%d_%d_%d_%d_%d" % (fam, ach, plus, comp, tbc)
                        _wrap_fn(lines, fn, os.path.join(gendir, body_file(
                            fam, kernel, plus, comp, tbc, tn, V, S)), comp, cltype)
                        regs.append("  rd_body[%d][%d][%d][%d][%d] = %s;" % (fam, ach, plus, comp, tbc, fn))
            fill = "rd_fill_body_%d_%d" % (fam, ach)
            emit("wrap_body_%d_%d.cpp" % (fam, ach), fill, lines, regs)
            parts.append(fill)
        lines, regs = ['#include "ref_driver.h"', ""], []
        for d in range(8):
            for plus in (0, 1):
                for comp in (0, 1):
                    for tbc in (0, 1):
                        fn = "u_%d_%d_%d_%d_%d" % (fam, d, plus, comp, tbc)
                        _wrap_fn(lines, fn, os.path.join(gendir, unpack_file(
                            fam, d, plus, comp, tbc, tn, V, S)), comp, cltype)
                        regs.append("  rd_unpack[%d][%d][%d][%d][%d] = %s;" % (fam, d, plus, comp, tbc, fn))
        fill = "rd_fill_unpack_%d" % fam
        emit("wrap_unpack_%d.cpp" % fam, fill, lines, regs)
        parts.append(fill)
        glue += ["void %s();" % q for q in parts]
        glue.append("void rd_fill_family%d() {" % fam)
        glue += ["  %s();" % q for q in parts]
        glue.append("}")
    lines, regs = glue + [""], []
    for d in range(8):
        for plus in (0, 1):
            fn = "p_%d_%d" % (d, plus)
            _wrap_fn(lines, fn, os.path.join(gendir, pack_file(d, plus, tn, V, S)), 1, "CloverBlock")
            regs.append("  rd_pack[%d][%d] = %s;" % (d, plus, fn))
    emit("wrap_faces.cpp", "rd_fill_faces", lines, regs)
    return files


def build(name, jobs=8, opt="-O2"):
    isa, prec, soa, lowprec = CONFIGS[name]
    V = VECLEN[(isa, prec)]
    tn = type_names(prec, lowprec)
    cfgdir = os.path.join(OUT, "build", name)
    os.makedirs(cfgdir, exist_ok=True)
    so = os.path.join(OUT, "libqphix_ref_%s.so" % name)
    if os.path.exists(so):
        return so
    # 1. generator
    with open(os.path.join(cfgdir, "output_dir.h"), "w") as f:
        f.write('#pragma once\n#include <string>\nstd::string output_dir = "%s";\n' % cfgdir)
    defs = ISA_DEFS[isa] + ["PRECISION=%d" % prec, "VECLEN=%d" % V, "SOALEN=%d" % soa]
    if lowprec:
        defs += ["ENABLE_LOW_PRECISION", "USE_LP_SPINOR", "USE_LP_GAUGE", "USE_LP_CLOVER"]
    srcs = sorted(os.path.join(REF, f) for f in os.listdir(REF) if f.endswith(".cc"))
    gen = os.path.join(cfgdir, "codegen")
    sh(["g++", "-O1", "-std=c++11", "-w", "-I" + cfgdir, "-I" + REF]
       + ["-D" + d for d in defs] + srcs + ["-o", gen])
    arch = isa
    gendir = os.path.join(cfgdir, "generated", arch, "generated")
    os.makedirs(gendir, exist_ok=True)
    sh([gen], cwd=cfgdir)
    # 2. wrappers
    wraps = write_wrappers(cfgdir, gendir, tn, V, soa)
    ft = "unsigned short" if lowprec else tn
    cflags = [opt, "-std=c++14", "-fPIC", "-fopenmp", "-w",
              "-I" + os.path.join(REF, "include"), "-I" + HERE,
              "-DRD_FT=" + ft, "-DRD_VEC=%d" % V, "-DRD_SOA=%d" % soa,
              "-DRD_HALF=%d" % (1 if lowprec else 0),
              "-DRD_AVX_UTILS=%d" % (1 if isa == "avx2" else 0)] + ISA_CFLAGS[isa]
    objs = []
    srcs = wraps + [os.path.join(HERE, "ref_driver.cpp")]
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = []
        for s in srcs:
            o = os.path.join(cfgdir, os.path.basename(s) + ".o")
            objs.append(o)
            futs.append(ex.submit(sh, ["g++"] + cflags + ["-c", s, "-o", o]))
        for fu in futs:
            fu.result()
    sh(["g++", "-shared", "-fopenmp", "-s", "-o", so] + objs)
    # the generated sources and objects are large; only the library is kept
    shutil.rmtree(cfgdir, ignore_errors=True)
    return so


def render_decls():
    """Render the reference's kernel declaration templates
    (codegen/jinja/{dslash,clov_dslash,tm_dslash,tm_clov_dslash}_decl.h.j2,
    unchanged, with jinja2 as codegen/jinja/generate_files.py does) and copy
    its Types<> header (codegen/include/decl_common.h) into
    oracle/_ref/include/, for the tests that compile a QPhiX-style caller
    against them and link the B200 library's per-tile kernels."""
    import jinja2
    inc = os.path.join(OUT, "include")
    os.makedirs(inc, exist_ok=True)
    env = jinja2.Environment(loader=jinja2.FileSystemLoader(REF))
    for k in ("dslash", "clov_dslash", "tm_dslash", "tm_clov_dslash"):
        text = env.get_template("jinja/%s_decl.h.j2" % k).render()
        with open(os.path.join(inc, "%s_decl.h" % k), "w") as f:
            f.write("#pragma once\n" + text)
    shutil.copy(os.path.join(REF, "include", "decl_common.h"), os.path.join(inc, "decl_common.h"))
    return inc


def main(argv):
    argv = list(argv)
    explicit = None
    if "--ref" in argv:
        i = argv.index("--ref")
        explicit = argv[i + 1]
        del argv[i:i + 2]
    root = reference_dir(explicit)
    if root is None:
        print("reference sources not present; using prebuilt oracle/_ref if any")
        return 0
    set_reference(root)
    print("rendered the reference's kernel declarations into", render_decls(), flush=True)
    names = argv or DEFAULT
    for n in names:
        print("building", n, "->", build(n), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
