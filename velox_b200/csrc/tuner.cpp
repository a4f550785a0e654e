// Launch-shape autotuner (tuner.h).
#include "tuner.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

namespace vxb {

namespace {

const char* kSiteNames[kTuneSiteCount] = {"collide_convex", "collide_complex", "collide_plane", "collide_any",
                                          "rewind_probe"};

// Candidate shapes (threads, blocks per SM). The collide kernels are built for
// at most 128 threads per block (255 registers: two 128-thread blocks fill an
// SM's register file), so their candidates trade block size against the grid
// cap: 2,048 threads per SM of grid (the fixed default, several waves that the
// block scheduler balances) or one resident wave (each thread walks several
// pairs). The probe kernel has the same register budget.
const LaunchShape kCandidates[kTuneCandidates] = {
    {128, 16}, {64, 32}, {32, 64}, {128, 2}, {64, 4}, {32, 8},
};

bool makeDirs(const std::string& file) {
    // mkdir -p of the file's directory
    std::string dir = file.substr(0, file.find_last_of('/'));
    if (dir.empty() || dir == file) return true;
    std::string part;
    std::stringstream ss(dir);
    std::string item;
    if (dir[0] == '/') part = "/";
    while (std::getline(ss, item, '/')) {
        if (item.empty()) continue;
        part += item + "/";
        struct stat st;
        if (stat(part.c_str(), &st) != 0 && mkdir(part.c_str(), 0755) != 0) return false;
    }
    return true;
}

}  // namespace

const char* Tuner::siteName(int site) {
    return site >= 0 && site < kTuneSiteCount ? kSiteNames[site] : "?";
}

LaunchShape Tuner::defaultShape(int) { return kCandidates[0]; }

LaunchShape Tuner::candidate(int, int k) { return kCandidates[k]; }

int Tuner::bucketOf(uint32_t items) {
    int b = 0;
    while (b < 31 && (items >> (b + 1)) != 0) ++b;
    return b;
}

void Tuner::init(int device, int smCount) {
    smCount_ = smCount;
    if (const char* m = std::getenv("VXB_TUNE")) mode_ = std::atoi(m) != 0 ? 1 : 0;
    cudaDeviceProp prop;
    std::memset(&prop, 0, sizeof(prop));
    cudaGetDeviceProperties(&prop, device);
    std::string name = prop.name;
    for (char& ch : name)
        if (ch == ' ' || ch == '\t') ch = '_';
    deviceKey_ = name + ":" + std::to_string(smCount) + ":" + std::to_string(prop.major) + "." +
                 std::to_string(prop.minor);
    if (const char* p = std::getenv("VXB_TUNE_CACHE")) {
        path_ = p;
    } else if (const char* x = std::getenv("XDG_CACHE_HOME"); x && *x) {
        path_ = std::string(x) + "/velox_b200/launch_shapes.txt";
    } else if (const char* h = std::getenv("HOME"); h && *h) {
        path_ = std::string(h) + "/.cache/velox_b200/launch_shapes.txt";
    }
    for (int s = 0; s < kTuneSiteCount; ++s) {
        cudaEventCreate(&start_[s]);
        cudaEventCreate(&stop_[s]);
    }
    ready_ = true;
    if (path_.empty()) return;
    std::ifstream in(path_);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string key, site;
        int bucket = -1;
        uint32_t threads = 0, bps = 0;
        if (!(ls >> key >> site >> bucket >> threads >> bps) || key != deviceKey_) continue;
        if (bucket < 0 || bucket >= kTuneBuckets) continue;
        for (int s = 0; s < kTuneSiteCount; ++s) {
            if (site != kSiteNames[s]) continue;
            for (int k = 0; k < kTuneCandidates; ++k)
                if (kCandidates[k].threads == threads && kCandidates[k].blocksPerSm == bps)
                    buckets_[s][bucket].decided = k;
        }
    }
}

void Tuner::release() {
    if (!ready_) return;
    for (int s = 0; s < kTuneSiteCount; ++s) harvest(s);
    if (dirty_) save();
    for (int s = 0; s < kTuneSiteCount; ++s) {
        if (start_[s]) cudaEventDestroy(start_[s]);
        if (stop_[s]) cudaEventDestroy(stop_[s]);
        start_[s] = stop_[s] = nullptr;
    }
    ready_ = false;
}

void Tuner::setMode(int mode) { mode_ = mode != 0 ? 1 : 0; }

// Folds a finished exploration sample of `site` into its bucket (non-blocking:
// a sample whose stop event has not completed stays pending).
void Tuner::harvest(int site) {
    Pending& p = pending_[site];
    if (!p.active) return;
    const cudaError_t q = cudaEventQuery(stop_[site]);
    if (q == cudaErrorNotReady) return;
    p.active = false;
    float ms = 0.0f;
    if (q != cudaSuccess || cudaEventElapsedTime(&ms, start_[site], stop_[site]) != cudaSuccess) {
        cudaGetLastError();  // a failed sample is dropped; the step's own status reports real errors
        return;
    }
    Bucket& b = buckets_[site][p.bucket];
    if (b.decided >= 0) return;
    const float perItem = ms / (float)(p.items ? p.items : 1);
    if (b.samples[p.cand] == 0 || perItem < b.bestPerItem[p.cand]) b.bestPerItem[p.cand] = perItem;
    ++b.samples[p.cand];
    for (int k = 0; k < kTuneCandidates; ++k)
        if (b.samples[k] < kTuneSamples) return;
    int best = 0;
    for (int k = 1; k < kTuneCandidates; ++k)
        if (b.bestPerItem[k] < b.bestPerItem[best]) best = k;
    b.decided = best;
    dirty_ = true;
    save();
}

LaunchShape Tuner::shapeFor(int site, uint32_t items, bool* decided) const {
    if (decided) *decided = false;
    if (site < 0 || site >= kTuneSiteCount) return kCandidates[0];
    if (mode_ == 0) {
        if (decided) *decided = true;
        return defaultShape(site);
    }
    const Bucket& b = buckets_[site][bucketOf(items)];
    if (b.decided >= 0) {
        if (decided) *decided = true;
        return kCandidates[b.decided];
    }
    return kCandidates[b.next];
}

TunedLaunch Tuner::begin(int site, uint32_t items, cudaStream_t stream) {
    TunedLaunch t;
    t.site = site;
    t.shape = defaultShape(site);
    if (!ready_ || mode_ == 0 || site < 0 || site >= kTuneSiteCount) return t;
    harvest(site);
    Bucket& b = buckets_[site][bucketOf(items)];
    if (b.decided >= 0) {
        t.shape = kCandidates[b.decided];
        return t;
    }
    if (pending_[site].active) return t;  // the previous sample is still in flight: launch the default, untimed
    // round-robin over the candidates that still need samples
    int k = b.next;
    for (int tries = 0; tries < kTuneCandidates && b.samples[k] >= kTuneSamples; ++tries) k = (k + 1) % kTuneCandidates;
    b.next = (k + 1) % kTuneCandidates;
    t.shape = kCandidates[k];
    if (cudaEventRecord(start_[site], stream) != cudaSuccess) {
        cudaGetLastError();
        return t;
    }
    t.timed = true;
    Pending& p = pending_[site];
    p.active = true;
    p.bucket = bucketOf(items);
    p.cand = k;
    p.items = items;
    return t;
}

void Tuner::end(const TunedLaunch& t, cudaStream_t stream) {
    if (!t.timed) return;
    if (cudaEventRecord(stop_[t.site], stream) != cudaSuccess) {
        cudaGetLastError();
        pending_[t.site].active = false;
    }
}

bool Tuner::save() {
    if (path_.empty() || deviceKey_.empty()) return false;
    std::vector<std::string> keep;
    {
        std::ifstream in(path_);
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream ls(line);
            std::string key;
            if ((ls >> key) && key != deviceKey_) keep.push_back(line);
        }
    }
    for (int s = 0; s < kTuneSiteCount; ++s)
        for (int bkt = 0; bkt < kTuneBuckets; ++bkt) {
            const int d = buckets_[s][bkt].decided;
            if (d < 0) continue;
            keep.push_back(deviceKey_ + " " + kSiteNames[s] + " " + std::to_string(bkt) + " " +
                           std::to_string(kCandidates[d].threads) + " " + std::to_string(kCandidates[d].blocksPerSm));
        }
    if (!makeDirs(path_)) return false;
    // write a sibling file and rename it over the cache, so readers never see half a file
    const std::string tmp = path_ + ".tmp." + std::to_string((long)getpid());
    {
        std::ofstream out(tmp, std::ios::trunc);
        if (!out) return false;
        out << "# velox_b200 launch shapes: device site log2(items) threads blocks_per_sm\n";
        for (const auto& l : keep)
            if (l.empty() || l[0] != '#') out << l << "\n";
        if (!out) return false;
    }
    if (std::rename(tmp.c_str(), path_.c_str()) != 0) {
        std::remove(tmp.c_str());
        return false;
    }
    dirty_ = false;
    return true;
}

}  // namespace vxb
