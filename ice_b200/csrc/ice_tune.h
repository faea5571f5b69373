// ice_tune.h -- the staged stage kernel's schedule per closure, as the tuner (ice_b200/tune.py) chose
// it by timing the kernel on one B200. Rewritten by the tuner; the library reads it at build time.
//
//   kz     the most planes one tile's chunk takes (its height is cut into equal chunks of at most kz,
//          fewer when that balances the last wave of CTAs better: choose_kz)
//   zpass  the passes of the CTA per plane that the tile-shape cost adds to the face tasks' passes
//          (the z face and the update): the larger, the more it favours few, full tiles
//   wcap   the widest tile, in owned columns
//
// The environment variable ICE_GPU_TUNE="kz,zpass,wcap" overrides the row of every closure (the
// tuner's sweep uses it).
//
// Measured: the first 8 blocks of the 48-block tree, 5401564 cells, one family at a time, FP32-flux form, 3 profiled steps. Stage-kernel launch in ms, the chosen row first:
//   MK: (16,1,16) 1.1808, (16,3,64) 1.1812, (16,2,64) 1.1816, (16,4,32) 1.1818, (16,1,32) 1.1818, (16,1,64) 1.1822; slowest (32,4,32) 1.2172
//   IG: (16,4,16) 1.1982, (16,4,64) 1.1987, (16,1,64) 1.1987, (16,3,64) 1.1992, (16,1,32) 1.1993, (16,2,16) 1.1993; slowest (32,1,32) 1.2460
//   AG: (32,1,24) 2.0126, (32,3,16) 2.0139, (24,4,24) 2.0145, (24,4,16) 2.0147, (24,3,32) 2.0147, (32,1,16) 2.0158; slowest (8,4,16) 2.1166
#pragma once

namespace ice {

struct TuneRow { int kz, zpass, wcap; };

// MK, IG, AG
constexpr TuneRow kTune[3] = {
    {16, 1, 16},
    {16, 4, 16},
    {32, 1, 24},
};

}  // namespace ice
