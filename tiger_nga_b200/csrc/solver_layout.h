// Layout of the generated solver tables (tiger_nga_b200/codegen.py: solver_tables).
// Hot tables (everything the right-hand side reads) are staged into shared memory per block;
// cold tables (the Jacobian's work lists) are read from global memory through L1. All tables
// are indexed by the slot's processing position p (falloff, exponential, constant).
#pragma once

namespace tng {

enum SvSize {
  SZ_NS, SZ_NV, SZ_NSLOT, SZ_NM, SZ_NFO, SZ_NFC, SZ_NCDCHUNK, SZ_NJDGRP, SZ_NGPAIR, SZ_NCDSTEP, SZ_NJDSTEP, SZ_COUNT
};
// hot doubles: plain-slot records (kSlotRec per plain slot, from position NFO: lnA|A, E, n),
// falloff (kFoRec: lnA0 E0 n0 lnAi Ei ni, pad), F_cent (kFcRec: a0 c0 a1 c1 a2 c2, pad), dense
// efficiencies (nm rows of eff_stride(ns)), thermo (ns rows of kThStride: hi 12, lo 12, pad),
// molar masses, their inverses, scalars.
// The record strides are odd: lanes that read the same field of consecutive records then hit 16
// distinct bank pairs per half-warp (an even stride such as 24 or 36 doubles puts eight lanes of a
// half-warp on one bank pair).
enum SvHd { HD_SLOT, HD_FO, HD_FC, HD_EFF, HD_TH, HD_WMOL, HD_INVW, HD_SCAL, HD_COUNT };
constexpr int kSlotRec = 3, kFoRec = 7, kFcRec = 7, kThStride = 25;
__host__ __device__ constexpr int eff_stride(int ns) { return ns | 1; }
// hot ints: slot words (2 per slot: flags|r0<<4|r1<<11|r2<<18, mw|fo<<8), falloff word
// (f0|f1<<4|(fc+1)<<8|m<<16), F_cent forms, chunks per species, and the production-rate terms
// interleaved by lane (step s of lane L at [s*32 + L]: nu | p<<8 | last-of-chunk<<20 | chunk<<21)
enum SvHi { HI_SLOT, HI_FO, HI_FC, HI_CD_SP_PTR, HI_CD_IL, HI_COUNT };
// cold ints: the Jacobian's mass-action terms interleaved by lane as int2 (x: p | other reactant
// a<<10 | other reactant b<<17 | third-body set<<24, 127 = none; y: nu | matrix offset<<8 |
// last-of-group<<20), and the third-body pairs (terms p<<12|kind<<8|nu)
enum SvCi { CI_JD_IL, CI_G_LANE_PTR, CI_G_LANE_LIST, CI_G_I, CI_G_M, CI_G_BEG, CI_G_END, CI_G_TERM, CI_COUNT };
enum SvScal { SC_RGAS, SC_TMID, SC_TN0, SC_TN1, SC_TC0, SC_TC1, SC_TD, SC_LNKMIN, SC_INVLN10 };
constexpr int kNone7 = 127;

struct SvLayout {
  int size[SZ_COUNT];
  int hd[HD_COUNT];
  int hi[HI_COUNT];
  int ci[CI_COUNT];
  int nhd, nhi, nci;
};

}  // namespace tng
