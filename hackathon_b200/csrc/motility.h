// Internal names of the decision layer (motility.cpp) over the public C ABI
// structs of include/ddm_b200.h.
#pragma once

#include <stdint.h>

#include "../../include/ddm_b200.h"

typedef ddm_radial_view mf_radial;
typedef ddm_motility_options mf_options;
typedef ddm_motility_fit mf_fit;
typedef ddm_motility_result mf_result;

enum {
  MF_MOTILE = 0,
  MF_NOT_MOTILE = 1,
  MF_DIRECTED_TRANSPORT = 2,
  MF_NO_DYNAMICS = 3,
  MF_UNLOCKED_EXPOSURE = 4
};

void mf_analyze_motility(const mf_radial *r, const mf_options *opt, mf_result *out);
