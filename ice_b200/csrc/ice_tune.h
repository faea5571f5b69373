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
//   MK: (24,4,64) 1.3244, (16,2,32) 1.3248, (16,4,32) 1.3252, (16,3,32) 1.3252, (16,4,64) 1.3254, (24,3,32) 1.3257; slowest (32,3,64) 1.3514
//   IG: (16,4,32) 1.3802, (16,3,64) 1.3803, (16,2,32) 1.3805, (16,4,16) 1.3807, (16,2,64) 1.3809, (16,4,64) 1.3810; slowest (8,4,64) 1.4076
//   AG: (32,4,32) 2.3719, (32,2,32) 2.3722, (32,3,16) 2.3727, (24,4,32) 2.3735, (24,3,32) 2.3735, (32,2,16) 2.3735; slowest (8,2,16) 2.4648
#pragma once

namespace ice {

struct TuneRow { int kz, zpass, wcap; };

// MK, IG, AG
constexpr TuneRow kTune[3] = {
    {24, 4, 64},
    {16, 4, 32},
    {32, 4, 32},
};

}  // namespace ice
