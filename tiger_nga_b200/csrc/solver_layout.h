// Layout of the generated solver tables (see tiger_nga_b200/codegen.py: solver_tables).
#pragma once

namespace tng {

enum SvSize { SZ_NS, SZ_NV, SZ_NSLOT, SZ_NM, SZ_NFO, SZ_NFC, SZ_NCDCHUNK, SZ_NJDGRP, SZ_NGPAIR, SZ_COUNT };
enum SvInt {
  I_SLOT_FLAGS, I_SLOT_REAC, I_SLOT_MW, I_SLOT_FO, I_FO_FLAGS, I_FO_FC, I_FO_M, I_FC_FORM, I_TB_PTR, I_TB_SP,
  I_CD_LANE_PTR, I_CD_LANE_LIST, I_CD_CHUNK_BEG, I_CD_CHUNK_END, I_CD_SLOT, I_CD_SP_PTR,
  I_JD_LANE_PTR, I_JD_LANE_LIST, I_JD_TGT, I_JD_BEG, I_JD_END, I_JD_SLOT, I_JD_POS,
  I_G_LANE_PTR, I_G_LANE_LIST, I_G_I, I_G_M, I_G_BEG, I_G_END, I_G_SLOT, I_G_KIND, I_COUNT
};
enum SvDbl {
  D_SLOT_A, D_SLOT_LNA, D_SLOT_N, D_SLOT_E, D_FO_PAR, D_FC_A, D_FC_C, D_TB_COEF, D_EFF, D_CD_NU, D_JD_NU, D_G_NU,
  D_TH_HI, D_TH_LO, D_WMOL, D_INVW, D_SCAL, D_COUNT
};
enum SvScal { SC_RGAS, SC_TMID, SC_TN0, SC_TN1, SC_TC0, SC_TC1, SC_TD, SC_LNKMIN, SC_INVLN10 };

struct SvLayout {
  int size[SZ_COUNT];
  int ioff[I_COUNT];
  int doff[D_COUNT];
  int nint, ndbl;
};

}  // namespace tng
