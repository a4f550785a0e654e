// Host-side check of the launch-shape cache file (velox_b200/csrc/tuner.cpp),
// built and run by tests/test_tuner_cache.py on a machine without a GPU: the
// tuner then launches fixed shapes, but decisions still reach the file.
//   tuner_cache_check <cache file>
#include <cstdio>
#include <cstdlib>

#include "tuner.h"

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    setenv("VXB_TUNE_CACHE", argv[1], 1);
    vxb::Tuner t;
    t.init(0, 148);
    t.beginTrials();
    t.decide(vxb::kTuneCollideConvex, 1u << 14);          // bucket 14: replaces the file's line
    t.decide(vxb::kTuneCollidePlane, (1u << 16) + 5u);     // bucket 16: a new line
    t.release();
    return 0;
}
