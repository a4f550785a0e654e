// Snapshots of the device-resident world (World::saveSnapshot /
// restoreSnapshot, src/world.cpp:2038-2128, for the state this library keeps
// on the device): every body array, the previous step's contacts and their
// keys (the warm-start cache, resting pairs' contacts included), the sleep
// state of every body and the last step's pair keys, the step and sleep
// configuration and the last step's statistics. Two forms:
//   * device slots: copies stay in device memory (device-to-device copies, no
//     host round trip) for rollback and replay;
//   * a byte image in caller memory (for files or another context that
//     loaded the same bodies).
// A snapshot restores only into a world with the same body count, world
// partition and geometry (shapes and their references into the soup, and the
// soup's array sizes: the image's body words index the destination's soup);
// restoring ends an active adjoint tape.
#include <cstring>

#include "context.cuh"

namespace vxb {

namespace {

constexpr uint32_t kSnapshotMagic = 0x53425856u;  // "VXBS"
constexpr uint32_t kSnapshotVersion = 3;

struct SnapshotHeader {
    uint32_t magic, version, n, worlds;
    uint32_t prevCount, cur, configured, stepContacts;
    uint32_t pairCount, sleepable, asleep, pad;
    uint64_t bodyBytes, totalBytes;
    uint64_t geometry;  // geometryKey of the world the image was taken from
    vxb_step_config config;
    vxb_sleep_config sleepConfig;
    vxb_step_stats stats;
};

// The loaded bodies' shape references and the soup's sizes in one key.
uint64_t geometryKey(const Context& c) { return c.bodyGeometryKey * 0x9e3779b97f4a7c15ull ^ c.soupGeometryKey; }

size_t bodyBytesOf(const Context& c) { return (((size_t)c.n * 16 + 255) & ~(size_t)255) * 16; }

size_t imageBytes(const Context& c, uint32_t prevCount, uint32_t pairCount) {
    return sizeof(SnapshotHeader) + bodyBytesOf(c) + (size_t)prevCount * (sizeof(vx_contact) + 8) +
           (size_t)c.n * 16 + (size_t)pairCount * 8;
}

SnapshotHeader headerOf(const Context& c) {
    SnapshotHeader h;
    std::memset(&h, 0, sizeof(h));
    h.magic = kSnapshotMagic;
    h.version = kSnapshotVersion;
    h.n = c.n;
    h.worlds = c.worlds;
    h.prevCount = c.prevCount;
    h.cur = (uint32_t)c.cur;
    h.configured = c.configured ? 1u : 0u;
    // a snapshot keeps the whole cache: after a restore, read-back of the last
    // step's contacts returns the cache (resting pairs' contacts included)
    h.stepContacts = c.prevCount;
    h.pairCount = c.sleep.pairCount;
    h.sleepable = c.sleep.sleepable;
    h.asleep = c.sleep.asleep;
    h.bodyBytes = bodyBytesOf(c);
    h.totalBytes = imageBytes(c, c.prevCount, c.sleep.pairCount);
    h.geometry = geometryKey(c);
    h.config = c.config;
    h.sleepConfig = c.sleep.config;
    h.stats = c.stats;
    return h;
}

#define VXB_TRY_SN(c, expr)            \
    do {                               \
        int s_ = (expr);               \
        if (s_ != VXB_OK) return s_;   \
    } while (0)

#define SN_CUDA(c, expr)                                              \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) return cudaStatus((c), e_, #expr);     \
    } while (0)

// Copies the world's state into `dst` (device or host memory, `kind` the
// direction) after the header.
int copyOut(Context& c, char* dst, cudaMemcpyKind kind) {
    const size_t bb = bodyBytesOf(c);
    SN_CUDA(c, cudaMemcpyAsync(dst, c.bodyBuf.ptr, bb, kind, c.stream));
    char* at = dst + bb;
    if (c.prevCount) {
        SN_CUDA(c, cudaMemcpyAsync(at, c.contactBuf[c.cur ^ 1].ptr, (size_t)c.prevCount * sizeof(vx_contact), kind,
                                   c.stream));
        at += (size_t)c.prevCount * sizeof(vx_contact);
        SN_CUDA(c, cudaMemcpyAsync(at, c.prevKeyBuf.ptr, (size_t)c.prevCount * 8, kind, c.stream));
        at += (size_t)c.prevCount * 8;
    }
    SN_CUDA(c, cudaMemcpyAsync(at, c.sleep.state.ptr, (size_t)c.n * 16, kind, c.stream));
    at += (size_t)c.n * 16;
    if (c.sleep.pairCount)
        SN_CUDA(c, cudaMemcpyAsync(at, c.sleep.pairs.ptr, (size_t)c.sleep.pairCount * 8, kind, c.stream));
    return VXB_OK;
}

int checkCompatible(Context& c, const SnapshotHeader& h) {
    if (h.magic != kSnapshotMagic || h.version != kSnapshotVersion)
        return fail(c, VXB_ERR_INVALID, "snapshot: not a snapshot image of this library version");
    if (h.n != c.n || h.worlds != c.worlds || h.bodyBytes != bodyBytesOf(c))
        return fail(c, VXB_ERR_INVALID, "snapshot: the world has another body count or world partition");
    if (h.geometry != geometryKey(c))
        return fail(c, VXB_ERR_INVALID, "snapshot: the world has other shapes or another soup");
    return VXB_OK;
}

// Restores from `src` (after the header) with header `h`.
int copyIn(Context& c, const SnapshotHeader& h, const char* src, cudaMemcpyKind kind) {
    const size_t bb = bodyBytesOf(c);
    tapeEnd(c);
    SN_CUDA(c, cudaMemcpyAsync(c.bodyBuf.ptr, src, bb, kind, c.stream));
    c.cur = (int)h.cur;
    if (h.prevCount) {
        VXB_TRY_SN(c, ensure(c, c.contactBuf[c.cur ^ 1], (size_t)h.prevCount * sizeof(vx_contact) + 128));
        VXB_TRY_SN(c, ensure(c, c.prevKeyBuf, (size_t)h.prevCount * 8 + 16));
        SN_CUDA(c, cudaMemcpyAsync(c.contactBuf[c.cur ^ 1].ptr, src + bb, (size_t)h.prevCount * sizeof(vx_contact),
                                   kind, c.stream));
        SN_CUDA(c, cudaMemcpyAsync(c.prevKeyBuf.ptr, src + bb + (size_t)h.prevCount * sizeof(vx_contact),
                                   (size_t)h.prevCount * 8, kind, c.stream));
    }
    const char* at = src + bb + (size_t)h.prevCount * (sizeof(vx_contact) + 8);
    VXB_TRY_SN(c, ensure(c, c.sleep.state, (size_t)c.n * 16 + 16));
    SN_CUDA(c, cudaMemcpyAsync(c.sleep.state.ptr, at, (size_t)c.n * 16, kind, c.stream));
    at += (size_t)c.n * 16;
    if (h.pairCount) {
        VXB_TRY_SN(c, ensure(c, c.sleep.pairs, (size_t)h.pairCount * 8 + 64));
        SN_CUDA(c, cudaMemcpyAsync(c.sleep.pairs.ptr, at, (size_t)h.pairCount * 8, kind, c.stream));
    }
    c.prevCount = h.prevCount;
    c.stepContacts = h.stepContacts;
    c.sleep.pairCount = h.pairCount;
    c.sleep.sleepable = h.sleepable;
    c.sleep.asleep = h.asleep;
    c.sleep.eventCount = 0;
    c.sleep.config = h.sleepConfig;
    c.config = h.config;
    c.configured = h.configured != 0;
    c.stats = h.stats;
    SN_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

}  // namespace

int snapshotSave(Context& c, uint32_t slot) {
    if (c.n == 0) return fail(c, VXB_ERR_INVALID, "snapshot: no bodies loaded");
    if (slot >= kSnapshotSlots) return fail(c, VXB_ERR_INVALID, "snapshot: slot out of range");
    DeviceSnapshot& s = c.snapshots[slot];
    const SnapshotHeader h = headerOf(c);
    const size_t payload = h.totalBytes - sizeof(SnapshotHeader);
    VXB_TRY_SN(c, ensure(c, s.buf, payload + 256));
    VXB_TRY_SN(c, copyOut(c, static_cast<char*>(s.buf.ptr), cudaMemcpyDeviceToDevice));
    static_assert(sizeof(SnapshotHeader) <= sizeof(s.header), "snapshot header storage");
    std::memcpy(s.header, &h, sizeof(h));
    s.valid = true;
    return VXB_OK;
}

int snapshotRestore(Context& c, uint32_t slot) {
    if (slot >= kSnapshotSlots || !c.snapshots[slot].valid)
        return fail(c, VXB_ERR_INVALID, "snapshot: no snapshot in this slot");
    SnapshotHeader h;
    std::memcpy(&h, c.snapshots[slot].header, sizeof(h));
    VXB_TRY_SN(c, checkCompatible(c, h));
    return copyIn(c, h, static_cast<const char*>(c.snapshots[slot].buf.ptr), cudaMemcpyDeviceToDevice);
}

int snapshotBytes(Context& c, size_t* bytes) {
    if (c.n == 0) return fail(c, VXB_ERR_INVALID, "snapshot: no bodies loaded");
    *bytes = imageBytes(c, c.prevCount, c.sleep.pairCount);
    return VXB_OK;
}

int snapshotRead(Context& c, void* out, size_t capacity) {
    if (c.n == 0) return fail(c, VXB_ERR_INVALID, "snapshot: no bodies loaded");
    const SnapshotHeader h = headerOf(c);
    if (capacity < h.totalBytes) return fail(c, VXB_ERR_CAPACITY, "snapshot: buffer too small");
    std::memcpy(out, &h, sizeof(h));
    VXB_TRY_SN(c, copyOut(c, static_cast<char*>(out) + sizeof(h), cudaMemcpyDeviceToHost));
    SN_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

int snapshotWrite(Context& c, const void* in, size_t size) {
    if (size < sizeof(SnapshotHeader)) return fail(c, VXB_ERR_INVALID, "snapshot: image too small");
    SnapshotHeader h;
    std::memcpy(&h, in, sizeof(h));
    VXB_TRY_SN(c, checkCompatible(c, h));
    if (size < h.totalBytes) return fail(c, VXB_ERR_INVALID, "snapshot: image truncated");
    return copyIn(c, h, static_cast<const char*>(in) + sizeof(h), cudaMemcpyHostToDevice);
}

}  // namespace vxb
