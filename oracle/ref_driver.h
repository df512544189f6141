// ref_driver.h -- shared declarations of the tile driver that runs the
// reference's generated per-tile kernels over a whole lattice (TEST
// INFRASTRUCTURE: built into oracle/_ref by oracle/ref_build.py, loaded only
// by tests/ and by bench.py's reference arm).
//
// Compile-time parameters (set by ref_build.py): RD_FT (float, double or
// unsigned short for the reference's `half`), RD_VEC, RD_SOA.
#pragma once

#include "decl_common.h" // the reference's Types<> (codegen/include/decl_common.h)
#if RD_AVX_UTILS
#include "avx_utils.h" // int->mask helpers the AVX/AVX2 bodies call (codegen/include/avx_utils.h)
#endif

typedef RD_FT FT;
typedef QPhiX::Types<FT, RD_VEC, RD_SOA, true>::FourSpinorBlock FSB;

// Every argument any generated body or face kernel refers to.  Each wrapper
// function copies the fields it needs into locals named as in the kernel
// signatures of codegen/jinja/*_decl.h.j2 and then includes the generated
// body.
struct TileArgs {
  const FSB *xyBase, *zbBase, *zfBase, *tbBase, *tfBase, *chiBase;
  FSB *oBase;
  const void *gBase;
  const void *clBase;
  const int *xbOffs, *xfOffs, *ybOffs, *yfOffs, *offs, *gOffs;
  const unsigned int *accumulate;
  FT coeff_s, coeff_t_f, coeff_t_b, alpha, mu, muinv, prec_mass_rho, beta;
  FT tbc_phases[4][2];
  FT *outbuf;
  const FT *inbuf;
  unsigned int mask;
  int dir;
};

typedef void (*TileFn)(const TileArgs &);

// [family 0..3][achimbdpsi][isPlus][compress12][tbc mask, bit mu = twisted in dim mu]
extern TileFn rd_body[4][2][2][2][16];
// [family][dir 0..7][isPlus][compress12][tbc]
extern TileFn rd_unpack[4][8][2][2][2];
// [dir][isPlus]
extern TileFn rd_pack[8][2];

void rd_fill_family0();
void rd_fill_family1();
void rd_fill_family2();
void rd_fill_family3();
void rd_fill_faces();
