// Launch-shape autotuner of the throughput kernels (narrow phase, rewind probe).
//
// Each tuned launch site picks its block size and its grid cap (blocks per SM,
// which sets how many pairs a thread walks in the grid-stride loop) per size
// bucket (floor(log2(items))). The first launch in an undecided bucket runs
// every candidate shape on the same inputs, twice, timed with CUDA events on
// the launching stream (the caller restores what a launch consumes before each
// trial), keeps the fastest, and then makes the real launch with it. Decisions
// are cached per device in a text file (one line per site and bucket) and read
// back by later contexts, which then launch the cached shape from their first
// call.
//
// The tuned kernels compute one pair per thread with no cross-thread state:
// their outputs are keyed by pair (records sorted by body pair afterwards), so
// the launch shape changes timing only, never a result.
//
// Environment: VXB_TUNE=0 launches the fixed default shapes (no trials, no
// cache); VXB_TUNE_CACHE=<file> names the cache file (empty: keep decisions in
// memory only); default $XDG_CACHE_HOME/velox_b200/launch_shapes.txt, else
// $HOME/.cache/velox_b200/launch_shapes.txt.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace vxb {

enum TuneSite : int {
    kTuneCollideConvex = 0,  // collideKernel over convex-convex pairs (GJK / EPA, clipping)
    kTuneCollideComplex,     // collideKernel over pairs with a mesh, heightfield or compound
    kTuneCollidePlane,       // collideKernel over body-plane pairs
    kTuneCollideAny,         // collideKernel over unclassified pairs (stage entry points)
    kTuneProbe,              // caProbeKernel: the rewind's end-of-step distance query per pair
    kTuneSiteCount
};

constexpr int kTuneBuckets = 33;     // floor(log2(items)) for items in [1, 2^32)
constexpr int kTuneCandidates = 6;   // shapes per site
constexpr int kTuneSamples = 2;      // trials per candidate before a decision

struct LaunchShape {
    uint32_t threads = 128;
    uint32_t blocksPerSm = 16;
    uint32_t grid(uint32_t items, int smCount) const {
        const uint64_t need = ((uint64_t)items + threads - 1) / threads;
        const uint64_t cap = (uint64_t)blocksPerSm * (uint64_t)smCount;
        const uint64_t g = need < cap ? need : cap;
        return (uint32_t)(g > 0 ? g : 1);
    }
};

class Tuner {
public:
    Tuner() {
        for (auto& site : decided_)
            for (int& d : site) d = -1;
    }
    // Reads the environment and the cache entries of this device.
    void init(int device, int smCount);
    // Destroys the events; writes pending decisions to the cache file.
    void release();
    // 0: fixed default shapes; 1: tune and use the cache.
    void setMode(int mode);
    int mode() const { return mode_; }

    // True when the size bucket of `items` at `site` has no shape yet: the
    // caller then times every candidate (trialStart / trialStop around each
    // launch) before its real launch.
    bool undecided(int site, uint32_t items) const;
    // Forgets the trial times of the previous bucket.
    void beginTrials();
    void trialStart(cudaStream_t stream);
    // Records the end of candidate k's trial and waits for it.
    cudaError_t trialStop(int k, cudaStream_t stream);
    // Keeps the candidate with the fastest trial for the bucket and writes
    // the cache file.
    void decide(int site, uint32_t items);

    // The shape the next launch of `site` over `items` uses, and whether that
    // bucket is decided (no trials left).
    LaunchShape shapeFor(int site, uint32_t items, bool* decided) const;
    // Writes this context's decisions into the cache file, merged with the
    // lines already there (other devices, and this device's buckets that this
    // context did not decide). Returns false when the file cannot be written.
    bool save();
    const std::string& cachePath() const { return path_; }

    static const char* siteName(int site);
    static LaunchShape defaultShape(int site);
    static LaunchShape candidate(int site, int k);

private:
    static int bucketOf(uint32_t items);

    int mode_ = 1;
    int smCount_ = 148;
    bool ready_ = false;
    bool dirty_ = false;
    std::string path_, deviceKey_;
    int decided_[kTuneSiteCount][kTuneBuckets];  // chosen candidate, -1 while undecided
    float trialMs_[kTuneCandidates] = {};        // best trial of each candidate (current bucket)
    cudaEvent_t start_ = nullptr, stop_ = nullptr;
};

}  // namespace vxb
