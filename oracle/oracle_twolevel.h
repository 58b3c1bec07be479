// Oracle (test infrastructure only): the two-level queries of
// oracle_twolevel.cpp for the other oracle files.
#pragma once

#include "oracle_scene.h"

namespace orc {

// Closest hit (t, u, v, global triangle id) and any hit over a two-level scene
// made by orc_two_level_new.
Hit two_level_closest(const void* two_level, V3 o, V3 d, float tmax);
bool two_level_any(const void* two_level, V3 o, V3 d, float tmax);

}  // namespace orc
