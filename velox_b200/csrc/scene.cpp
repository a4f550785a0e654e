// Synthetic benchmark scenes and body construction (host code).
//
// vxb_scene_generate() emits shape-level specs (vx_shape_spec) for the five
// benchmark workloads, seeded with std::mt19937_64. vxb_bodies_from_specs()
// turns specs into vx_body records plus the convex-hull soup, following the
// reference's World::add* construction rules (src/world.cpp:646-985,
// :1305-1318): the same mass/inertia formulas, body defaults and CCD defaults
// (WorldCcdDefaults, include/velox/ccd.h:98-105). Hull topology and mass
// properties are computed here by a brute-force convex hull and a
// tetrahedral mass integral with a Jacobi eigen-solve (the reference uses
// QuickHull, src/mass_properties.h; triangulation may differ, the solid does
// not).
#include "velox_b200.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <random>
#include <unordered_map>
#include <vector>

namespace {

struct Rng {
    std::mt19937_64 engine;
    explicit Rng(uint64_t seed) : engine(seed) {}
    double u01() { return double(engine() >> 11) * (1.0 / 9007199254740992.0); }
    float uniform(float lo, float hi) { return float(lo + (hi - lo) * u01()); }
    float normal(float sigma) {  // Box-Muller
        double u1 = u01(), u2 = u01();
        if (u1 < 1e-300) u1 = 1e-300;
        return float(sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
    }
    vx_quat quaternion() {  // uniform random rotation (Shoemake)
        double u1 = u01(), u2 = u01(), u3 = u01();
        double a = std::sqrt(1.0 - u1), b = std::sqrt(u1);
        double t1 = 6.283185307179586 * u2, t2 = 6.283185307179586 * u3;
        vx_quat q{float(a * std::sin(t1)), float(a * std::cos(t1)), float(b * std::sin(t2)),
                  float(b * std::cos(t2))};
        float len = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        q.x /= len; q.y /= len; q.z /= len; q.w /= len;
        return q;
    }
};

vx_shape_spec baseSpec(uint8_t shape, uint32_t world) {
    vx_shape_spec s;
    std::memset(&s, 0, sizeof(s));
    s.shape = shape;
    s.world = world;
    s.enableSleep = 0;  // benchmark scenes: every body is simulated every step
    s.orientation = {0, 0, 0, 1};
    s.friction = 0.5f;
    s.restitution = 0.3f;
    s.planeNormal = {0, 1, 0};
    return s;
}

vx_shape_spec planeSpec(uint32_t world) { return baseSpec(VX_SHAPE_PLANE, world); }

constexpr float kPi = 3.14159265358979f;
constexpr float kDensity = 1000.0f;

// Bounding radius used for rejection sampling.
float boundRadius(const vx_shape_spec& s, const vx_vec3* pool) {
    switch (s.shape) {
    case VX_SHAPE_SPHERE: return s.radius;
    case VX_SHAPE_BOX:
        return std::sqrt(s.halfExtents.x * s.halfExtents.x + s.halfExtents.y * s.halfExtents.y +
                         s.halfExtents.z * s.halfExtents.z);
    case VX_SHAPE_CAPSULE: return s.radius + s.halfHeight;
    case VX_SHAPE_CYLINDER: return std::sqrt(s.radius * s.radius + s.halfHeight * s.halfHeight);
    case VX_SHAPE_HULL: {
        float r = 0;
        for (uint32_t i = 0; i < s.hullCount; ++i) {
            const vx_vec3& p = pool[s.hullFirst + i];
            r = std::max(r, std::sqrt(p.x * p.x + p.y * p.y + p.z * p.z));
        }
        return r;
    }
    default: return 0;
    }
}

// Spatial hash of placed bounding spheres for non-overlap rejection sampling.
struct Placer {
    float cell;
    std::unordered_map<uint64_t, std::vector<std::array<float, 4>>> grid;
    explicit Placer(float c) : cell(c) {}
    static uint64_t key(int x, int y, int z) {
        return (uint64_t(uint32_t(x + (1 << 20))) << 42) ^ (uint64_t(uint32_t(y + (1 << 20))) << 21) ^
               uint64_t(uint32_t(z + (1 << 20)));
    }
    bool free(float x, float y, float z, float r) const {
        int cx = int(std::floor(x / cell)), cy = int(std::floor(y / cell)), cz = int(std::floor(z / cell));
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    auto it = grid.find(key(cx + dx, cy + dy, cz + dz));
                    if (it == grid.end()) continue;
                    for (const auto& s : it->second) {
                        float ddx = s[0] - x, ddy = s[1] - y, ddz = s[2] - z, rr = s[3] + r;
                        if (ddx * ddx + ddy * ddy + ddz * ddz < rr * rr) return false;
                    }
                }
        return true;
    }
    void add(float x, float y, float z, float r) {
        int cx = int(std::floor(x / cell)), cy = int(std::floor(y / cell)), cz = int(std::floor(z / cell));
        grid[key(cx, cy, cz)].push_back({x, y, z, r});
    }
};

// Random body of the mixed-shape distribution: spheres r~U[0.2,0.5]; boxes
// half extents ~U[0.2,0.6]; capsules r~U[0.15,0.3], half height ~U[0.2,0.5];
// cylinders r~U[0.2,0.4], half height ~U[0.2,0.5]; hulls of 16 points on
// ellipsoids with semi-axes ~U[0.3,0.7]. Mass = 1000 kg/m^3 * volume.
vx_shape_spec randomShape(Rng& rng, uint8_t shape, uint32_t world, std::vector<vx_vec3>& pool) {
    vx_shape_spec s = baseSpec(shape, world);
    switch (shape) {
    case VX_SHAPE_SPHERE:
        s.radius = rng.uniform(0.2f, 0.5f);
        s.mass = kDensity * (4.0f / 3.0f) * kPi * s.radius * s.radius * s.radius;
        break;
    case VX_SHAPE_BOX:
        s.halfExtents = {rng.uniform(0.2f, 0.6f), rng.uniform(0.2f, 0.6f), rng.uniform(0.2f, 0.6f)};
        s.mass = kDensity * 8.0f * s.halfExtents.x * s.halfExtents.y * s.halfExtents.z;
        break;
    case VX_SHAPE_CAPSULE:
        s.radius = rng.uniform(0.15f, 0.3f);
        s.halfHeight = rng.uniform(0.2f, 0.5f);
        s.mass = kDensity * (kPi * s.radius * s.radius * 2.0f * s.halfHeight +
                             (4.0f / 3.0f) * kPi * s.radius * s.radius * s.radius);
        break;
    case VX_SHAPE_CYLINDER:
        s.radius = rng.uniform(0.2f, 0.4f);
        s.halfHeight = rng.uniform(0.2f, 0.5f);
        s.mass = kDensity * kPi * s.radius * s.radius * 2.0f * s.halfHeight;
        break;
    case VX_SHAPE_HULL: {
        float ax = rng.uniform(0.3f, 0.7f), ay = rng.uniform(0.3f, 0.7f), az = rng.uniform(0.3f, 0.7f);
        s.hullFirst = (uint32_t)pool.size();
        s.hullCount = 16;
        for (int i = 0; i < 16; ++i) {
            float x, y, z, l;
            do {
                x = rng.normal(1.0f); y = rng.normal(1.0f); z = rng.normal(1.0f);
                l = std::sqrt(x * x + y * y + z * z);
            } while (l < 1e-3f);
            pool.push_back({ax * x / l, ay * y / l, az * z / l});
        }
        s.mass = 0.0f;  // filled from the hull volume below
        break;
    }
    }
    return s;
}

}  // namespace

// --- convex hull + mass properties --------------------------------------

namespace {

struct D3 { double x, y, z; };
D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
D3 crs(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double dt3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Brute-force hull of a small point set in general position: every triple
// with all remaining points strictly on one side is an outward face.
bool hullTriangles(const std::vector<D3>& p, std::vector<std::array<uint32_t, 3>>& tris) {
    const size_t n = p.size();
    double scale = 0;
    for (auto& q : p) scale = std::max(scale, std::sqrt(dt3(q, q)));
    const double eps = 1e-9 * scale * scale * scale + 1e-15;
    tris.clear();
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = i + 1; j < n; ++j)
            for (uint32_t k = j + 1; k < n; ++k) {
                D3 nrm = crs(sub(p[j], p[i]), sub(p[k], p[i]));
                if (dt3(nrm, nrm) < 1e-24) continue;
                int pos = 0, neg = 0;
                for (uint32_t m = 0; m < n && !(pos && neg); ++m) {
                    if (m == i || m == j || m == k) continue;
                    double s = dt3(nrm, sub(p[m], p[i]));
                    if (s > eps) ++pos;
                    else if (s < -eps) ++neg;
                    else { pos = neg = 1; }  // coplanar fourth point: not general position
                }
                if (pos && neg) continue;
                if (pos) tris.push_back({i, k, j});  // others above: flip to face outward
                else tris.push_back({i, j, k});
            }
    return tris.size() >= 4;
}

void jacobiEigen(double a[3][3], double evals[3], double v[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) v[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (off < 1e-30) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (std::fabs(a[p][q]) < 1e-300) continue;
                double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {  // A <- A J
                    double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {  // A <- J^T A
                    double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = c * vkp - s * vkq;
                    v[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 3; ++i) evals[i] = a[i][i];
}

vx_quat quatFromMatrix(double m[3][3]) {  // columns are the rotated basis
    double tr = m[0][0] + m[1][1] + m[2][2];
    double x, y, z, w;
    if (tr > 0) {
        double s = std::sqrt(tr + 1.0) * 2;
        w = 0.25 * s; x = (m[2][1] - m[1][2]) / s; y = (m[0][2] - m[2][0]) / s; z = (m[1][0] - m[0][1]) / s;
    } else if (m[0][0] > m[1][1] && m[0][0] > m[2][2]) {
        double s = std::sqrt(1.0 + m[0][0] - m[1][1] - m[2][2]) * 2;
        w = (m[2][1] - m[1][2]) / s; x = 0.25 * s; y = (m[0][1] + m[1][0]) / s; z = (m[0][2] + m[2][0]) / s;
    } else if (m[1][1] > m[2][2]) {
        double s = std::sqrt(1.0 + m[1][1] - m[0][0] - m[2][2]) * 2;
        w = (m[0][2] - m[2][0]) / s; x = (m[0][1] + m[1][0]) / s; y = 0.25 * s; z = (m[1][2] + m[2][1]) / s;
    } else {
        double s = std::sqrt(1.0 + m[2][2] - m[0][0] - m[1][1]) * 2;
        w = (m[1][0] - m[0][1]) / s; x = (m[0][2] + m[2][0]) / s; y = (m[1][2] + m[2][1]) / s; z = 0.25 * s;
    }
    double l = std::sqrt(x * x + y * y + z * z + w * w);
    return {float(x / l), float(y / l), float(z / l), float(w / l)};
}

struct HullProps {
    double volume;
    D3 center;
    double moments[3];
    vx_quat frame;
    std::vector<std::array<uint32_t, 3>> tris;
};

bool hullProperties(const std::vector<D3>& pts, HullProps& out) {
    if (!hullTriangles(pts, out.tris)) return false;
    D3 ref{0, 0, 0};
    for (auto& p : pts) { ref.x += p.x; ref.y += p.y; ref.z += p.z; }
    ref.x /= pts.size(); ref.y /= pts.size(); ref.z /= pts.size();
    double vol = 0, cx = 0, cy = 0, cz = 0;
    double C[3][3] = {{0}};  // second moments about ref: integral of r r^T
    for (auto& t : out.tris) {
        D3 a = sub(pts[t[0]], ref), b = sub(pts[t[1]], ref), c = sub(pts[t[2]], ref);
        double v6 = dt3(a, crs(b, c));
        double v = v6 / 6.0;
        vol += v;
        cx += v * (a.x + b.x + c.x) / 4.0;
        cy += v * (a.y + b.y + c.y) / 4.0;
        cz += v * (a.z + b.z + c.z) / 4.0;
        double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, Cc[3] = {c.x, c.y, c.z};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                C[i][j] += v / 20.0 * (2 * (A[i] * A[j] + B[i] * B[j] + Cc[i] * Cc[j]) +
                                       A[i] * B[j] + A[j] * B[i] + A[i] * Cc[j] + A[j] * Cc[i] +
                                       B[i] * Cc[j] + B[j] * Cc[i]);
    }
    if (!(vol > 0)) return false;
    D3 com{cx / vol, cy / vol, cz / vol};
    double M[3] = {com.x, com.y, com.z};
    for (int i = 0; i < 3; ++i)  // shift second moments to the centre of mass
        for (int j = 0; j < 3; ++j) C[i][j] -= vol * M[i] * M[j];
    double tr = C[0][0] + C[1][1] + C[2][2];
    double I[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) I[i][j] = (i == j ? tr : 0.0) - C[i][j];
    double evec[3][3];
    jacobiEigen(I, out.moments, evec);
    double det = evec[0][0] * (evec[1][1] * evec[2][2] - evec[1][2] * evec[2][1]) -
                 evec[0][1] * (evec[1][0] * evec[2][2] - evec[1][2] * evec[2][0]) +
                 evec[0][2] * (evec[1][0] * evec[2][1] - evec[1][1] * evec[2][0]);
    if (det < 0)
        for (int k = 0; k < 3; ++k) evec[k][2] = -evec[k][2];
    out.frame = quatFromMatrix(evec);
    out.volume = vol;
    out.center = {ref.x + com.x, ref.y + com.y, ref.z + com.z};
    return true;
}

void defaultBody(vx_body& b) {  // velox::Body defaults (body.h:128-171) + addBody CCD defaults
    std::memset(&b, 0, sizeof(b));
    b.orientation = {0, 0, 0, 1};
    b.invMass = 1.0f;
    b.inertiaOrientation = {0, 0, 0, 1};
    b.restitution = 0.3f;
    b.friction = 0.5f;
    b.frictionScale = {1, 1, 1};
    b.frictionCombine = VX_COMBINE_GEOMETRIC_MEAN;
    b.restitutionCombine = VX_COMBINE_MINIMUM;
    b.gravityScale = 1.0f;
    b.motionType = VX_MOTION_DYNAMIC;
    b.ccdTuning.quality = VX_QUALITY_MEDIUM;
    b.ccdTuning.collisionMargin = 0.0f;
    b.ccdTuning.speculativeDistance = 0.01f;
    b.ccdTuning.enableContinuous = 1;
    b.ccdTuning.minVelocityForCCD = 1.0f;
    b.ccdTuning.ccdSettings.quality = 1;  // CcdQuality::Balanced preset (ccd.h:43-53)
    b.ccdTuning.ccdSettings.maxAdvancementIterations = 16;
    b.ccdTuning.ccdSettings.maxRootFindIterations = 12;
    b.ccdTuning.ccdSettings.distanceTolerance = 1e-3f;
    b.ccdTuning.ccdSettings.timeTolerance = 1e-5f;
    b.ccdTuning.ccdSettings.enableRotationalCcd = 1;
    b.ccdTuning.ccdSettings.enableCompoundCcd = 1;
    b.ccdTuning.ccdSettings.useBrentRootFinder = 1;
    b.ccdTuning.ccdSettings.meshBvhMaxDepth = 8;
    b.ccdTuning.ccdSettings.speculativeMargin = 0.01f;
    b.geometryQuality = VX_GEOM_NORMAL;
    b.categoryBits = 1u;
    b.maskBits = 0xffffffffu;
    b.enableSleep = 1;
    b.shape = VX_SHAPE_SPHERE;
    b.radius = 0.5f;
    b.halfExtents = {0.5f, 0.5f, 0.5f};
    b.capsuleHalfHeight = 0.5f;
    b.planeNormal = {0, 1, 0};
}

}  // namespace

extern "C" {

int vxb_scene_generate(int config, uint64_t seed, uint32_t size, vx_shape_spec* specs,
                       uint32_t cap, uint32_t* count, vx_vec3* pool, uint32_t poolCap,
                       uint32_t* poolCount) {
    Rng rng(seed);
    std::vector<vx_shape_spec> out;
    std::vector<vx_vec3> pts;
    switch (config) {
    case 1: {  // 1,000 unit-mass boxes (half 0.5) on a 10x10x10 lattice, 1.1 m pitch
        const int side = size ? (int)size : 10;
        out.push_back(planeSpec(0));
        for (int j = 0; j < side; ++j)
            for (int i = 0; i < side; ++i)
                for (int k = 0; k < side; ++k) {
                    vx_shape_spec s = baseSpec(VX_SHAPE_BOX, 0);
                    s.halfExtents = {0.5f, 0.5f, 0.5f};
                    s.mass = 1.0f;
                    s.friction = 0.5f;
                    s.restitution = 0.0f;
                    s.position = {(i - 0.5f * (side - 1)) * 1.1f + rng.uniform(-0.05f, 0.05f),
                                  1.5f + j * 1.1f + rng.uniform(-0.05f, 0.05f),
                                  (k - 0.5f * (side - 1)) * 1.1f + rng.uniform(-0.05f, 0.05f)};
                    s.orientation = rng.quaternion();
                    out.push_back(s);
                }
        break;
    }
    case 2: {  // mixed shapes in a 200 x 200 x 60 m box above the plane
        const uint32_t n = size ? size : 100000u;
        const float half = 100.0f * std::sqrt(float(n) / 100000.0f);
        out.push_back(planeSpec(0));
        Placer placer(2.5f);
        for (uint32_t b = 0; b < n; ++b) {
            float u = rng.uniform(0.0f, 1.0f);
            uint8_t shape = u < 0.25f ? VX_SHAPE_SPHERE : u < 0.5f ? VX_SHAPE_BOX
                          : u < 0.7f ? VX_SHAPE_CAPSULE : u < 0.8f ? VX_SHAPE_CYLINDER : VX_SHAPE_HULL;
            vx_shape_spec s = randomShape(rng, shape, 0, pts);
            float r = boundRadius(s, pts.data());
            for (int attempt = 0; attempt < 10000; ++attempt) {
                float x = rng.uniform(-half, half), y = rng.uniform(1.0f, 61.0f), z = rng.uniform(-half, half);
                if (y - r < 0.05f) continue;
                if (!placer.free(x, y, z, r)) continue;
                placer.add(x, y, z, r);
                s.position = {x, y, z};
                break;
            }
            s.orientation = rng.quaternion();
            s.velocity = {rng.normal(2.0f), rng.normal(2.0f), rng.normal(2.0f)};
            out.push_back(s);
        }
        break;
    }
    case 3: {  // 20-row unit-box pyramids on a 16 x 16 grid, 30 m apart
        const uint32_t pyramids = size ? size : 256u;
        const int rows = 20;
        out.push_back(planeSpec(0));
        for (uint32_t p = 0; p < pyramids; ++p) {
            float cx = (float(p % 16) - 7.5f) * 30.0f, cz = (float(p / 16) - 7.5f) * 30.0f;
            for (int k = 0; k < rows; ++k)
                for (int i = 0; i < rows - k; ++i) {
                    vx_shape_spec s = baseSpec(VX_SHAPE_BOX, 0);
                    s.halfExtents = {0.5f, 0.5f, 0.5f};
                    s.mass = 1.0f;
                    s.friction = 0.6f;
                    s.position = {cx + (i - 0.5f * (rows - k - 1)) * 1.002f + rng.uniform(-1e-3f, 1e-3f),
                                  0.5f + float(k), cz + rng.uniform(-1e-3f, 1e-3f)};
                    out.push_back(s);
                }
        }
        break;
    }
    case 4: {  // batched worlds: plane + log-uniform [8,512] spheres/boxes/capsules
        const uint32_t worlds = size ? size : 4096u;
        for (uint32_t w = 0; w < worlds; ++w) {
            int bodies = (int)std::lround(std::exp(rng.uniform(std::log(8.0f), std::log(512.0f))));
            out.push_back(planeSpec(w));
            const float half = 0.75f * std::sqrt(float(bodies)) + 1.0f;
            Placer placer(2.5f);
            for (int b = 0; b < bodies; ++b) {
                int kind = (int)(rng.u01() * 3.0);
                uint8_t shape = kind == 0 ? VX_SHAPE_SPHERE : kind == 1 ? VX_SHAPE_BOX : VX_SHAPE_CAPSULE;
                vx_shape_spec s = randomShape(rng, shape, w, pts);
                float r = boundRadius(s, nullptr);
                for (int attempt = 0; attempt < 10000; ++attempt) {
                    float x = rng.uniform(-half, half), y = rng.uniform(1.0f, 10.0f), z = rng.uniform(-half, half);
                    if (y - r < 0.05f) continue;
                    if (!placer.free(x, y, z, r)) continue;
                    placer.add(x, y, z, r);
                    s.position = {x, y, z};
                    break;
                }
                s.orientation = rng.quaternion();
                out.push_back(s);
            }
        }
        break;
    }
    case 5: {  // differentiation worlds: 5-box stack + sphere projectile
        const uint32_t worlds = size ? size : 1024u;
        for (uint32_t w = 0; w < worlds; ++w) {
            out.push_back(planeSpec(w));
            for (int k = 0; k < 5; ++k) {
                vx_shape_spec s = baseSpec(VX_SHAPE_BOX, w);
                s.halfExtents = {0.5f, 0.5f, 0.5f};
                s.mass = 1.0f;
                s.position = {0.0f, 0.5f + float(k), 0.0f};
                out.push_back(s);
            }
            vx_shape_spec s = baseSpec(VX_SHAPE_SPHERE, w);
            s.radius = 0.3f;
            s.mass = 2.0f;
            s.position = {-6.0f, rng.uniform(0.5f, 4.0f), 0.0f};
            s.velocity = {rng.uniform(4.0f, 12.0f), 0.0f, 0.0f};
            out.push_back(s);
        }
        break;
    }
    default:
        return VXB_ERR_INVALID;
    }
    // Hull masses come from their volumes (density 1000 kg/m^3).
    for (auto& s : out)
        if (s.shape == VX_SHAPE_HULL) {
            std::vector<D3> p;
            for (uint32_t i = 0; i < s.hullCount; ++i) {
                const vx_vec3& q = pts[s.hullFirst + i];
                p.push_back({q.x, q.y, q.z});
            }
            HullProps props;
            if (!hullProperties(p, props)) return VXB_ERR_INVALID;
            s.mass = float(kDensity * props.volume);
        }
    if (count) *count = (uint32_t)out.size();
    if (poolCount) *poolCount = (uint32_t)pts.size();
    if (specs && out.size() > cap) return VXB_ERR_CAPACITY;
    if (pool && pts.size() > poolCap) return VXB_ERR_CAPACITY;
    if (specs) std::memcpy(specs, out.data(), out.size() * sizeof(vx_shape_spec));
    if (pool) std::memcpy(pool, pts.data(), pts.size() * sizeof(vx_vec3));
    return VXB_OK;
}

int vxb_bodies_from_specs(const vx_shape_spec* specs, uint32_t n, const vx_vec3* pool,
                          vx_body* bodies, vx_vec3* hullPoints, uint32_t hullCap,
                          uint32_t* hullCount, uint32_t* faceIndices, uint32_t faceCap,
                          uint32_t* faceIndexCount) {
    uint32_t hp = 0, fi = 0;
    int status = VXB_OK;
    for (uint32_t k = 0; k < n; ++k) {
        const vx_shape_spec& s = specs[k];
        vx_body b;
        defaultBody(b);
        const float mass = s.mass;
        b.position = s.position;
        b.motionType = mass > 0.0f ? VX_MOTION_DYNAMIC : VX_MOTION_STATIC;
        b.invMass = mass > 0.0f ? 1.0f / mass : 0.0f;
        switch (s.shape) {
        case VX_SHAPE_SPHERE:  // world.cpp:741-757
            b.shape = VX_SHAPE_SPHERE;
            b.radius = s.radius;
            if (mass > 0.0f) {
                float i = 0.4f * mass * s.radius * s.radius;
                b.invInertia = {1.0f / i, 1.0f / i, 1.0f / i};
            }
            break;
        case VX_SHAPE_BOX: {  // world.cpp:759-780
            b.shape = VX_SHAPE_BOX;
            b.halfExtents = s.halfExtents;
            if (mass > 0.0f) {
                float ex = s.halfExtents.x * 2.0f, ey = s.halfExtents.y * 2.0f, ez = s.halfExtents.z * 2.0f;
                float kk = mass / 12.0f;
                b.invInertia = {1.0f / (kk * (ey * ey + ez * ez)), 1.0f / (kk * (ex * ex + ez * ez)),
                                1.0f / (kk * (ex * ex + ey * ey))};
            }
            break;
        }
        case VX_SHAPE_CAPSULE: {  // world.cpp:782-815
            b.shape = VX_SHAPE_CAPSULE;
            b.radius = s.radius;
            b.capsuleHalfHeight = s.halfHeight;
            if (mass > 0.0f) {
                float r = s.radius, hh = s.halfHeight;
                float cylinderWeight = 2.0f * hh;
                float sphereWeight = (4.0f / 3.0f) * r;
                float cylinderMass = mass * cylinderWeight / (cylinderWeight + sphereWeight);
                float sphereMass = mass - cylinderMass;
                float iy = 0.5f * cylinderMass * r * r + 0.4f * sphereMass * r * r;
                float ix = cylinderMass * (3.0f * r * r + 4.0f * hh * hh) / 12.0f +
                           sphereMass * (0.4f * r * r + 0.75f * hh * r + hh * hh);
                b.invInertia = {1.0f / ix, 1.0f / iy, 1.0f / ix};
            }
            break;
        }
        case VX_SHAPE_CYLINDER: {  // world.cpp:817-838
            b.shape = VX_SHAPE_CYLINDER;
            b.radius = s.radius;
            b.capsuleHalfHeight = s.halfHeight;
            if (mass > 0.0f) {
                float height = 2.0f * s.halfHeight;
                float iy = 0.5f * mass * s.radius * s.radius;
                float ix = mass * (3.0f * s.radius * s.radius + height * height) / 12.0f;
                b.invInertia = {1.0f / ix, 1.0f / iy, 1.0f / ix};
            }
            break;
        }
        case VX_SHAPE_PLANE: {  // world.cpp:1305-1318
            b.shape = VX_SHAPE_PLANE;
            b.motionType = VX_MOTION_STATIC;
            float l = std::sqrt(s.planeNormal.x * s.planeNormal.x + s.planeNormal.y * s.planeNormal.y +
                                s.planeNormal.z * s.planeNormal.z);
            float inv = l > 1e-8f ? 1.0f / l : 0.0f;
            b.planeNormal = {s.planeNormal.x * inv, s.planeNormal.y * inv, s.planeNormal.z * inv};
            b.planeOffset = s.planeOffset;
            b.invMass = 0.0f;
            b.position = {0, 0, 0};
            break;
        }
        case VX_SHAPE_HULL: {  // world.cpp:909-985, own hull + mass integration
            std::vector<D3> p;
            for (uint32_t i = 0; i < s.hullCount; ++i) {
                const vx_vec3& q = pool[s.hullFirst + i];
                p.push_back({q.x, q.y, q.z});
            }
            HullProps props;
            if (!hullProperties(p, props)) return VXB_ERR_INVALID;
            b.shape = VX_SHAPE_HULL;
            D3 c = mass > 0.0f ? props.center : D3{0, 0, 0};
            b.position = {float(s.position.x + c.x), float(s.position.y + c.y), float(s.position.z + c.z)};
            b.hullFirst = hp;
            b.hullCount = s.hullCount;
            b.hullFaceFirst = fi;
            b.hullFaceCount = (uint32_t)props.tris.size();
            float r2 = 0.0f;
            for (uint32_t i = 0; i < s.hullCount; ++i) {
                vx_vec3 q{float(p[i].x - c.x), float(p[i].y - c.y), float(p[i].z - c.z)};
                if (hullPoints && hp < hullCap) hullPoints[hp] = q;
                ++hp;
                r2 = std::max(r2, q.x * q.x + q.y * q.y + q.z * q.z);
            }
            for (const auto& t : props.tris)
                for (int e = 0; e < 3; ++e) {
                    if (faceIndices && fi < faceCap) faceIndices[fi] = t[e];
                    ++fi;
                }
            b.radius = std::sqrt(r2);
            if (mass > 0.0f) {
                float density = mass / float(props.volume);
                b.invInertia = {1.0f / float(props.moments[0] * density),
                                1.0f / float(props.moments[1] * density),
                                1.0f / float(props.moments[2] * density)};
                b.inertiaOrientation = props.frame;
            }
            break;
        }
        default:
            return VXB_ERR_UNSUPPORTED;
        }
        if (s.shape != VX_SHAPE_PLANE) {
            b.orientation = s.orientation;
            b.velocity = s.velocity;
            b.angularVelocity = s.angularVelocity;
            b.friction = s.friction;
            b.restitution = s.restitution;
            b.enableSleep = s.enableSleep;
        }
        if (bodies) bodies[k] = b;
    }
    if (hullCount) *hullCount = hp;
    if (faceIndexCount) *faceIndexCount = fi;
    if ((hullPoints && hp > hullCap) || (faceIndices && fi > faceCap)) status = VXB_ERR_CAPACITY;
    return status;
}

}  // extern "C"
