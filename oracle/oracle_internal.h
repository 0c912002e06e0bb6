// oracle_internal.h -- C++ helpers shared between the oracle's files.
// TEST INFRASTRUCTURE ONLY (see vrad_oracle.h).
#pragma once

#include "vrad_oracle.h"

struct OrcKd {
    const orc_kdnode *nodes;
    const int32_t *indices;
    const orc_tri *tris;
    float bounds[6];
};

bool orc_kd_segment_blocked(const OrcKd &kd, const orc_ray &r, bool sky_pass);
