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
#pragma once

namespace ice {

struct TuneRow { int kz, zpass, wcap; };

// MK, IG, AG. Defaults until a tuning run replaces them.
constexpr TuneRow kTune[3] = {
    {32, 2, 64},
    {32, 2, 64},
    {32, 2, 32},
};

}  // namespace ice
