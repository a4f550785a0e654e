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
    for (auto& site : decided_)
        for (int& d : site) d = -1;
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
    if (cudaEventCreate(&start_) != cudaSuccess || cudaEventCreate(&stop_) != cudaSuccess) {
        cudaGetLastError();
        mode_ = 0;  // no events: fixed shapes
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
                if (kCandidates[k].threads == threads && kCandidates[k].blocksPerSm == bps) decided_[s][bucket] = k;
        }
    }
}

void Tuner::release() {
    if (!ready_) return;
    if (dirty_) save();
    if (start_) cudaEventDestroy(start_);
    if (stop_) cudaEventDestroy(stop_);
    start_ = stop_ = nullptr;
    ready_ = false;
}

void Tuner::setMode(int mode) { mode_ = mode != 0 && start_ && stop_ ? 1 : 0; }

bool Tuner::undecided(int site, uint32_t items) const {
    return ready_ && mode_ == 1 && site >= 0 && site < kTuneSiteCount && decided_[site][bucketOf(items)] < 0;
}

void Tuner::beginTrials() {
    for (float& t : trialMs_) t = -1.0f;
}

void Tuner::trialStart(cudaStream_t stream) { cudaEventRecord(start_, stream); }

cudaError_t Tuner::trialStop(int k, cudaStream_t stream) {
    float ms = 0.0f;
    cudaError_t e = cudaEventRecord(stop_, stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(stop_);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, start_, stop_);
    if (e != cudaSuccess) return e;
    if (trialMs_[k] < 0.0f || ms < trialMs_[k]) trialMs_[k] = ms;
    return cudaSuccess;
}

void Tuner::decide(int site, uint32_t items) {
    int best = 0;
    for (int k = 1; k < kTuneCandidates; ++k)
        if (trialMs_[k] >= 0.0f && (trialMs_[best] < 0.0f || trialMs_[k] < trialMs_[best])) best = k;
    decided_[site][bucketOf(items)] = best;
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
    const int d = decided_[site][bucketOf(items)];
    if (d >= 0) {
        if (decided) *decided = true;
        return kCandidates[d];
    }
    return defaultShape(site);
}

bool Tuner::save() {
    if (path_.empty() || deviceKey_.empty()) return false;
    std::vector<std::string> keep;
    {
        // keep every line this context does not replace: other devices' lines,
        // and this device's buckets decided by other contexts
        std::ifstream in(path_);
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream ls(line);
            std::string key, site;
            int bucket = -1;
            if (!(ls >> key)) continue;
            bool replaced = false;
            if (key == deviceKey_ && (ls >> site >> bucket) && bucket >= 0 && bucket < kTuneBuckets)
                for (int s = 0; s < kTuneSiteCount; ++s)
                    if (site == kSiteNames[s] && decided_[s][bucket] >= 0) replaced = true;
            if (!replaced) keep.push_back(line);
        }
    }
    for (int s = 0; s < kTuneSiteCount; ++s)
        for (int bkt = 0; bkt < kTuneBuckets; ++bkt) {
            const int d = decided_[s][bkt];
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
