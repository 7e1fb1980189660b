// Tuning knobs of the Laplace passes and the autotuner's JSON cache.
//
// The knobs change launch shapes only (tile sizes, staging variant, stream
// overlap, points per lane), never the arithmetic: every setting gives the
// same outputs.  A tuned setting is stored per problem signature in a JSON
// file written by fmmlib3d_b200/autotune.py; single calls and plans look their
// signature up when their tree is built.  Cache file, in order: the path given
// to fmm3d_set_tuning_cache, the environment variable FMM3D_TUNING_CACHE, or
// tuning_cache.json next to libfmm3d_b200.so.  An empty path or "none"
// disables the cache.
#pragma once
#include <string>

namespace fmm {

// 0 = automatic for every knob
struct TuneKnobs {
    int m2l_kt = 0;       // M2L targets per tile
    int trans_kt = 0;     // M2M / L2L targets per tile
    int tc_variant = 0;   // tensor-core M2L staging: 1 = 16-wide K chunks x 3 stages, 2 = 32-wide x 2
    int overlap = 0;      // 1 = near field concurrent with the far field, 2 = all passes in order
    int p2p_ept = 0;      // mixed-form P2P: at most 1, 2 or 4 evaluation points per lane
};
constexpr int kNumKnobs = 5;

inline void knobs_to_array(const TuneKnobs &k, int *a)
{
    a[0] = k.m2l_kt; a[1] = k.trans_kt; a[2] = k.tc_variant; a[3] = k.overlap; a[4] = k.p2p_ept;
}
inline TuneKnobs knobs_from_array(const int *a)
{
    TuneKnobs k;
    k.m2l_kt = a[0]; k.trans_kt = a[1]; k.tc_variant = a[2]; k.overlap = a[3]; k.p2p_ept = a[4];
    return k;
}

// The knobs stored for this signature, if the cache has them.
bool tuning_lookup(const std::string &signature, TuneKnobs &k);

// "<device name>/<SM count>" of the current device (part of every signature).
std::string device_tag();

// round(log2(n)), 0 for n <= 0 (signature buckets)
int log2_bucket(long long n);

}  // namespace fmm
