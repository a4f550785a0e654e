/*
 * Test infrastructure (not the product): an FP64 CPU restatement of the
 * device world's step with its contact set frozen, and its hand-derived
 * reverse (adjoint). It is the FP64 reference the GPU adjoint kernel is
 * checked against, and the function the FP64 central finite differences
 * differentiate.
 *
 * The reference engine has no adjoint. The step restated here is its own
 * (World::stepImpl, src/world.cpp:4007-4397, with the CUDA backend's coloured
 * solve, src/backend_cuda.cu:569-761):
 *   prepare     orientation normalisation and first-substep velocity
 *               integration (backend_cuda.cu:80-89)
 *   substeps    s > 0: velocity integration; s == 0: warm start
 *               (src/narrowphase.h:80-124); 2*velocityIterations colour-major
 *               sweeps of solveContact (narrowphase.h:130-366, two-axis
 *               friction); Body::advanceTransform (include/velox/body.h:266-321,
 *               isotropic inertia)
 *   correction  positionIterations colour-major passes of the split-impulse
 *               position correction (world.cpp:4370-4397)
 * with, per step, the contacts (normal, anchors, bias0, coefficients), their
 * colours, the warm-start sources (the previous step's contact whose impulses
 * a contact inherits, world.cpp:4133-4184) and the restitution-reference
 * sources frozen from the forward pass. A contact's approach speed vn0 is its
 * relative normal velocity at its anchors at detection, or the frozen
 * source's vn0; on the first step, a vn0 carried from before the recorded
 * steps is the recorded constant. The conservative-advancement rewind is not
 * part of the model (a world that rewound is not smooth).
 *
 * Everything is double precision; bodies must have isotropic inverse inertia.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "velox_b200_types.h"

typedef struct { double x, y, z; } D3;
typedef struct { double x, y, z, w; } D4;

static D3 d3(double x, double y, double z) { D3 r = {x, y, z}; return r; }
static D3 add(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
static D3 sub(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
static D3 mul(D3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
static double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static D3 cross(D3 a, D3 b) { return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static void acc(D3* a, D3 b) { a->x += b.x; a->y += b.y; a->z += b.z; }
static void accs(D3* a, D3 b, double s) { a->x += b.x * s; a->y += b.y * s; a->z += b.z * s; }
static D3 fromf(vx_vec3 v) { return d3(v.x, v.y, v.z); }

/* rotate(q, v) = v + 2 qv x (qv x v + w v)   (include/velox/math.h:104-109) */
static D3 rot(D4 q, D3 v) {
    D3 qv = d3(q.x, q.y, q.z);
    D3 u = add(cross(qv, v), mul(v, q.w));
    return add(v, mul(cross(qv, u), 2.0));
}
/* reverse of rot: accumulates dL/dq into qb, dL/dv into vb given ob = dL/dout */
static void rotRev(D4 q, D3 v, D3 ob, D4* qb, D3* vb) {
    D3 qv = d3(q.x, q.y, q.z);
    D3 u = add(cross(qv, v), mul(v, q.w));
    D3 tb = mul(ob, 2.0);                  /* t = qv x u */
    D3 qvb = cross(u, tb);                 /* d(qv x u)/dqv */
    D3 ub = cross(tb, qv);                 /* d(qv x u)/du */
    acc(&qvb, cross(v, ub));               /* u = qv x v + w v */
    if (vb) { acc(vb, ob); acc(vb, cross(ub, qv)); accs(vb, ub, q.w); }
    qb->w += dot(ub, v);
    qb->x += qvb.x; qb->y += qvb.y; qb->z += qvb.z;
}

static D4 qnormalize(D4 q, double* lenOut) {
    double len = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (lenOut) *lenOut = len;
    D4 r = {q.x / len, q.y / len, q.z / len, q.w / len};
    return r;
}
/* reverse of q/|q|: in = q (before), ob = dL/dout -> returns dL/dq */
static D4 qnormalizeRev(D4 q, D4 ob) {
    double len;
    D4 n = qnormalize(q, &len);
    double d = n.x * ob.x + n.y * ob.y + n.z * ob.z + n.w * ob.w;
    D4 r = {(ob.x - n.x * d) / len, (ob.y - n.y * d) / len, (ob.z - n.z * d) / len, (ob.w - n.w * d) / len};
    return r;
}

/* integrate(q, w, h) = normalize(q + (w h/2, 0) (x) q)   (math.h:115-118) */
static D4 qraw(D4 q, D3 w, double h) {
    double ax = w.x * 0.5 * h, ay = w.y * 0.5 * h, az = w.z * 0.5 * h;
    D4 dq = {ax * q.w + ay * q.z - az * q.y, -ax * q.z + ay * q.w + az * q.x, ax * q.y - ay * q.x + az * q.w,
             -ax * q.x - ay * q.y - az * q.z};
    D4 r = {q.x + dq.x, q.y + dq.y, q.z + dq.z, q.w + dq.w};
    return r;
}
static D4 qintegrate(D4 q, D3 w, double h) { return qnormalize(qraw(q, w, h), NULL); }
static void qintegrateRev(D4 q, D3 w, double h, D4 ob, D4* qb, D3* wb) {
    D4 rb = qnormalizeRev(qraw(q, w, h), ob);
    double ax = w.x * 0.5 * h, ay = w.y * 0.5 * h, az = w.z * 0.5 * h;
    /* raw = q + dq(a, q) */
    qb->x += rb.x; qb->y += rb.y; qb->z += rb.z; qb->w += rb.w;
    /* dq.x = ax qw + ay qz - az qy ; dq.y = -ax qz + ay qw + az qx ;
       dq.z = ax qy - ay qx + az qw ; dq.w = -ax qx - ay qy - az qz */
    double axb = rb.x * q.w - rb.y * q.z + rb.z * q.y - rb.w * q.x;
    double ayb = rb.x * q.z + rb.y * q.w - rb.z * q.x - rb.w * q.y;
    double azb = -rb.x * q.y + rb.y * q.x + rb.z * q.w - rb.w * q.z;
    qb->w += rb.x * ax + rb.y * ay + rb.z * az;
    qb->z += rb.x * ay - rb.y * ax - rb.w * az;
    qb->y += -rb.x * az + rb.z * ax - rb.w * ay;
    qb->x += rb.y * az - rb.z * ay - rb.w * ax;
    wb->x += axb * 0.5 * h; wb->y += ayb * 0.5 * h; wb->z += azb * 0.5 * h;
}

/* contactTangents (src/narrowphase.h:38-50): frozen with the normal. */
static void tangents(D3 n, D3* t1, D3* t2) {
    D3 an = d3(fabs(n.x), fabs(n.y), fabs(n.z));
    D3 r = an.x < an.y ? (an.x < an.z ? d3(1, 0, 0) : d3(0, 0, 1)) : (an.y < an.z ? d3(0, 1, 0) : d3(0, 0, 1));
    D3 c = cross(n, r);
    double l = sqrt(dot(c, c));
    *t1 = l > 1e-8 ? mul(c, 1.0 / l) : d3(0, 0, 0);
    *t2 = cross(n, *t1);
}

/* ---- bodies ---------------------------------------------------------------- */

typedef struct {
    int dyn, stat, locked, rotLocked, sensor, asleep, sphere;
    double gs, ld, ad;
} Prop;

typedef struct { D3 p; D4 q; D3 v, w; } St;



typedef struct {
    double dt, gx, gy, gz;
    int substeps, sweeps, positionIterations, stackStabilization;
    double stackStiffness, stackDamping;
} adjref_config;

static Prop propOf(const vx_body* b) {
    Prop p;
    p.dyn = b->motionType == VX_MOTION_DYNAMIC;
    p.stat = b->motionType == VX_MOTION_STATIC;
    p.locked = b->ccdTuning.quality == VX_QUALITY_LOCKED;
    p.rotLocked = p.locked || b->fixedRotation;
    p.sensor = b->sensor != 0;
    p.asleep = b->asleep != 0;
    p.sphere = b->shape == VX_SHAPE_SPHERE;
    p.gs = b->gravityScale;
    p.ld = b->linearDamping;
    p.ad = b->angularDamping;
    return p;
}

/* ---- rows ------------------------------------------------------------------- */

typedef struct {
    int a, b, solved;
    D3 n, t1, t2, la, lb;
    double bias0, e, f1, f2;
    double vn0;  /* as recorded (the constant a first-step carried vn0 takes) */
    int color;
} Row;

typedef struct {  /* pose terms of one row at one substep */
    D3 ra, rb, raxn, rbxn, raxt1, rbxt1, raxt2, rbxt2;
    double ma, mb, iA, iB, kN, k1, k2, gap, target0;
    int gpos;  /* the live gap's branch: positive (speculative target) */
} Prep;

typedef struct {  /* adjoints of the pose terms */
    D3 ra, rb, raxn, rbxn, raxt1, rbxt1, raxt2, rbxt2;
    double kN, k1, k2, target0;
} PrepBar;

typedef struct {
    const Prop* prop;
    const double* invMass;
    const double* invI;
    double* gInvMass;
    double* gInvI;
} Mass;

static double solverInvMass(const Mass* M, int i) {
    return M->prop[i].dyn && !M->prop[i].locked ? M->invMass[i] : 0.0;
}
static double isoInvI(const Mass* M, int i) { return M->prop[i].dyn && !M->prop[i].rotLocked ? M->invI[i] : 0.0; }
static void addInvMass(const Mass* M, int i, double g) { if (M->prop[i].dyn && !M->prop[i].locked) M->gInvMass[i] += g; }
static void addInvI(const Mass* M, int i, double g) { if (M->prop[i].dyn && !M->prop[i].rotLocked) M->gInvI[i] += g; }

static D3 anchorArm(const Prop* P, D4 q, D3 local) { return P->sphere ? local : rot(q, local); }

static void prep(const Mass* M, const St* S, const Row* r, double h, Prep* P) {
    const St* A = &S[r->a];
    const St* B = &S[r->b];
    P->ra = anchorArm(&M->prop[r->a], A->q, r->la);
    P->rb = anchorArm(&M->prop[r->b], B->q, r->lb);
    P->ma = solverInvMass(M, r->a);
    P->mb = solverInvMass(M, r->b);
    P->iA = isoInvI(M, r->a);
    P->iB = isoInvI(M, r->b);
    P->raxn = cross(P->ra, r->n);
    P->rbxn = cross(P->rb, r->n);
    P->raxt1 = cross(P->ra, r->t1); P->rbxt1 = cross(P->rb, r->t1);
    P->raxt2 = cross(P->ra, r->t2); P->rbxt2 = cross(P->rb, r->t2);
    P->kN = P->ma + P->mb + P->iA * dot(P->raxn, P->raxn) + P->iB * dot(P->rbxn, P->rbxn);
    P->k1 = P->ma + P->mb + P->iA * dot(P->raxt1, P->raxt1) + P->iB * dot(P->rbxt1, P->rbxt1);
    P->k2 = P->ma + P->mb + P->iA * dot(P->raxt2, P->raxt2) + P->iB * dot(P->rbxt2, P->rbxt2);
    P->gap = r->bias0 + dot(r->n, sub(add(A->p, P->ra), add(B->p, P->rb)));
    P->gpos = P->gap > 0.0;
    P->target0 = P->gpos ? -P->gap / h : 0.0;
}

/* reverse of prep: pose-term adjoints -> state and mass adjoints */
static void prepRev(const Mass* M, const St* S, const Row* r, double h, const Prep* P, PrepBar* Pb, D3* pb, D4* qb) {
    const int a = r->a, b = r->b;
    /* effective masses */
    addInvMass(M, a, Pb->kN + Pb->k1 + Pb->k2);
    addInvMass(M, b, Pb->kN + Pb->k1 + Pb->k2);
    addInvI(M, a, Pb->kN * dot(P->raxn, P->raxn) + Pb->k1 * dot(P->raxt1, P->raxt1) + Pb->k2 * dot(P->raxt2, P->raxt2));
    addInvI(M, b, Pb->kN * dot(P->rbxn, P->rbxn) + Pb->k1 * dot(P->rbxt1, P->rbxt1) + Pb->k2 * dot(P->rbxt2, P->rbxt2));
    accs(&Pb->raxn, P->raxn, 2.0 * P->iA * Pb->kN);
    accs(&Pb->rbxn, P->rbxn, 2.0 * P->iB * Pb->kN);
    accs(&Pb->raxt1, P->raxt1, 2.0 * P->iA * Pb->k1);
    accs(&Pb->rbxt1, P->rbxt1, 2.0 * P->iB * Pb->k1);
    accs(&Pb->raxt2, P->raxt2, 2.0 * P->iA * Pb->k2);
    accs(&Pb->rbxt2, P->rbxt2, 2.0 * P->iB * Pb->k2);
    /* cross products r x d: d(r x d)/dr adjoint = d x bar */
    acc(&Pb->ra, cross(r->n, Pb->raxn));
    acc(&Pb->ra, cross(r->t1, Pb->raxt1));
    acc(&Pb->ra, cross(r->t2, Pb->raxt2));
    acc(&Pb->rb, cross(r->n, Pb->rbxn));
    acc(&Pb->rb, cross(r->t1, Pb->rbxt1));
    acc(&Pb->rb, cross(r->t2, Pb->rbxt2));
    /* live gap */
    double gapb = P->gpos ? -Pb->target0 / h : 0.0;
    accs(&pb[a], r->n, gapb);
    accs(&Pb->ra, r->n, gapb);
    accs(&pb[b], r->n, -gapb);
    accs(&Pb->rb, r->n, -gapb);
    /* arms */
    if (!M->prop[a].sphere) rotRev(S[a].q, r->la, Pb->ra, &qb[a], NULL);
    if (!M->prop[b].sphere) rotRev(S[b].q, r->lb, Pb->rb, &qb[b], NULL);
}

/* branch bits of one row update */
enum { BR_RESTITUTION = 1, BR_RESMAX = 2, BR_CLAMP = 4, BR_FRICTION = 8, BR_M1 = 16, BR_M2 = 32, BR_ELLIPSE = 64,
       BR_SKIP = 128 };

typedef struct { D3 va, wa, vb, wb; double ln, l1, l2; int bits; } RowIn;

static void applyImpulse(St* A, St* B, const Prep* P, D3 imp, D3 raxI, D3 rbxI, int dynA, int dynB) {
    if (dynA) { accs(&A->v, imp, P->ma); accs(&A->w, raxI, P->iA); }
    if (dynB) { accs(&B->v, imp, -P->mb); accs(&B->w, rbxI, -P->iB); }
}

/* one solveContact sweep (two-axis friction) on prepared terms; lam[3] in/out.
 * forced >= 0: take the branch decisions from those bits (BR_*) instead of
 * deciding them (the piece another run took). */
static void rowForward(const Mass* M, St* S, const Row* r, const Prep* P, double vn0, double* lam, RowIn* tape,
                       int forced) {
    St* A = &S[r->a];
    St* B = &S[r->b];
    const int dynA = M->prop[r->a].dyn, dynB = M->prop[r->b].dyn;
    if (tape) {
        tape->va = A->v; tape->wa = A->w; tape->vb = B->v; tape->wb = B->w;
        tape->ln = lam[0]; tape->l1 = lam[1]; tape->l2 = lam[2]; tape->bits = 0;
    }
    if (P->kN <= 0.0) { if (tape) tape->bits = BR_SKIP; return; }
    const int F = forced >= 0;
    int bits = 0;
    double vn = dot(r->n, sub(A->v, B->v)) + dot(P->raxn, A->w) - dot(P->rbxn, B->w);
    double target = P->target0;
    if (F ? (forced & BR_RESTITUTION) != 0 : (vn0 < -1.0 && (!P->gpos || vn > 0.0))) {
        bits |= BR_RESTITUTION;
        double rest = -r->e * vn0;
        if (F ? (forced & BR_RESMAX) != 0 : rest > target) { target = rest; bits |= BR_RESMAX; }
    }
    double jn = (target - vn) / P->kN;
    double s = lam[0] + jn;
    const int clamp = F ? (forced & BR_CLAMP) != 0 : s > 0.0;
    double lnp = clamp ? s : 0.0;
    if (clamp) bits |= BR_CLAMP;
    double dn = lnp - lam[0];
    lam[0] = lnp;
    applyImpulse(A, B, P, mul(r->n, dn), mul(P->raxn, dn), mul(P->rbxn, dn), dynA, dynB);
    if (P->k1 > 0.0 && P->k2 > 0.0) {
        bits |= BR_FRICTION;
        double rv1 = dot(r->t1, sub(A->v, B->v)) + dot(P->raxt1, A->w) - dot(P->rbxt1, B->w);
        double rv2 = dot(r->t2, sub(A->v, B->v)) + dot(P->raxt2, A->w) - dot(P->rbxt2, B->w);
        double u1 = lam[1] - rv1 / P->k1, u2 = lam[2] - rv2 / P->k2;
        double m1 = r->f1 * lnp, m2 = r->f2 * lnp;
        const int on1 = F ? (forced & BR_M1) != 0 : m1 > 0.0, on2 = F ? (forced & BR_M2) != 0 : m2 > 0.0;
        if (on1) bits |= BR_M1; else u1 = 0.0;
        if (on2) bits |= BR_M2; else u2 = 0.0;
        double E = (on1 ? u1 * u1 / (m1 * m1) : 0.0) + (on2 ? u2 * u2 / (m2 * m2) : 0.0);
        if (F ? (forced & BR_ELLIPSE) != 0 : E > 1.0) {
            bits |= BR_ELLIPSE;
            double sc = 1.0 / sqrt(E);
            u1 *= sc; u2 *= sc;
        }
        double d1 = u1 - lam[1], d2 = u2 - lam[2];
        lam[1] = u1; lam[2] = u2;
        D3 imp = add(mul(r->t1, d1), mul(r->t2, d2));
        applyImpulse(A, B, P, imp, add(mul(P->raxt1, d1), mul(P->raxt2, d2)),
                     add(mul(P->rbxt1, d1), mul(P->rbxt2, d2)), dynA, dynB);
    }
    if (tape) tape->bits = bits;
}

/* reverse of rowForward. Sb holds velocity adjoints (v, w) after the row and is
 * updated to before it; lamb[3] likewise; Pb accumulates pose-term adjoints,
 * vn0b the restitution reference's adjoint. Branches replay from the tape. */
static void rowReverse(const Mass* M, const Row* r, const Prep* P, double vn0, const RowIn* in, D3* vbA, D3* wbA,
                       D3* vbB, D3* wbB, double* lamb, PrepBar* Pb, double* vn0b) {
    const int bits = in->bits;
    if (bits & BR_SKIP) return;
    const int dynA = M->prop[r->a].dyn, dynB = M->prop[r->b].dyn;
    /* forward replay */
    D3 va = in->va, wa = in->wa, vb = in->vb, wb = in->wb;
    double vn = dot(r->n, sub(va, vb)) + dot(P->raxn, wa) - dot(P->rbxn, wb);
    double target = (bits & BR_RESMAX) ? -r->e * vn0 : P->target0;
    double jn = (target - vn) / P->kN;
    double s = in->ln + jn;
    double lnp = (bits & BR_CLAMP) ? s : 0.0;
    double dn = lnp - in->ln;
    D3 va1 = va, wa1 = wa, vb1 = vb, wb1 = wb;
    if (dynA) { accs(&va1, r->n, P->ma * dn); accs(&wa1, P->raxn, P->iA * dn); }
    if (dynB) { accs(&vb1, r->n, -P->mb * dn); accs(&wb1, P->rbxn, -P->iB * dn); }
    double lnpb = lamb[0], l1b = 0.0, l2b = 0.0;
    D3 VA = *vbA, WA = *wbA, VB = *vbB, WB = *wbB;  /* adjoints after the row */
    if (bits & BR_FRICTION) {
        double rv1 = dot(r->t1, sub(va1, vb1)) + dot(P->raxt1, wa1) - dot(P->rbxt1, wb1);
        double rv2 = dot(r->t2, sub(va1, vb1)) + dot(P->raxt2, wa1) - dot(P->rbxt2, wb1);
        double u1 = in->l1 - rv1 / P->k1, u2 = in->l2 - rv2 / P->k2;
        double m1 = r->f1 * lnp, m2 = r->f2 * lnp;
        double z1 = (bits & BR_M1) ? u1 : 0.0, z2 = (bits & BR_M2) ? u2 : 0.0;
        double E = ((bits & BR_M1) ? z1 * z1 / (m1 * m1) : 0.0) + ((bits & BR_M2) ? z2 * z2 / (m2 * m2) : 0.0);
        double sc = (bits & BR_ELLIPSE) ? 1.0 / sqrt(E) : 1.0;
        double y1 = z1 * sc, y2 = z2 * sc;
        double d1 = y1 - in->l1, d2 = y2 - in->l2;
        /* impulse application (16) */
        double d1b = 0.0, d2b = 0.0;
        D3 imp = add(mul(r->t1, d1), mul(r->t2, d2));
        D3 raxI = add(mul(P->raxt1, d1), mul(P->raxt2, d2));
        D3 rbxI = add(mul(P->rbxt1, d1), mul(P->rbxt2, d2));
        if (dynA) {
            d1b += P->ma * dot(r->t1, VA) + P->iA * dot(P->raxt1, WA);
            d2b += P->ma * dot(r->t2, VA) + P->iA * dot(P->raxt2, WA);
            addInvMass(M, r->a, dot(imp, VA));
            addInvI(M, r->a, dot(raxI, WA));
            accs(&Pb->raxt1, WA, P->iA * d1);
            accs(&Pb->raxt2, WA, P->iA * d2);
        }
        if (dynB) {
            d1b -= P->mb * dot(r->t1, VB) + P->iB * dot(P->rbxt1, WB);
            d2b -= P->mb * dot(r->t2, VB) + P->iB * dot(P->rbxt2, WB);
            addInvMass(M, r->b, -dot(imp, VB));
            addInvI(M, r->b, -dot(rbxI, WB));
            accs(&Pb->rbxt1, WB, -P->iB * d1);
            accs(&Pb->rbxt2, WB, -P->iB * d2);
        }
        /* (14) d = y - l */
        double y1b = lamb[1] + d1b, y2b = lamb[2] + d2b;
        l1b -= d1b;
        l2b -= d2b;
        /* (13) ellipse scaling */
        double z1b = y1b * sc, z2b = y2b * sc, Eb = 0.0;
        if (bits & BR_ELLIPSE) {
            double scb = z1 * y1b + z2 * y2b;
            Eb = scb * (-0.5) * pow(E, -1.5);
        }
        /* (12) */
        double m1b = 0.0, m2b = 0.0;
        if (bits & BR_M1) { z1b += Eb * 2.0 * z1 / (m1 * m1); m1b += Eb * (-2.0 * z1 * z1 / (m1 * m1 * m1)); }
        if (bits & BR_M2) { z2b += Eb * 2.0 * z2 / (m2 * m2); m2b += Eb * (-2.0 * z2 * z2 / (m2 * m2 * m2)); }
        /* (11) */
        double u1b = (bits & BR_M1) ? z1b : 0.0, u2b = (bits & BR_M2) ? z2b : 0.0;
        /* (10) */
        lnpb += r->f1 * m1b + r->f2 * m2b;
        /* (9) */
        l1b += u1b;
        l2b += u2b;
        double rv1b = -u1b / P->k1, rv2b = -u2b / P->k2;
        Pb->k1 += u1b * rv1 / (P->k1 * P->k1);
        Pb->k2 += u2b * rv2 / (P->k2 * P->k2);
        /* (8) */
        accs(&VA, r->t1, rv1b); accs(&VA, r->t2, rv2b);
        accs(&WA, P->raxt1, rv1b); accs(&WA, P->raxt2, rv2b);
        accs(&VB, r->t1, -rv1b); accs(&VB, r->t2, -rv2b);
        accs(&WB, P->rbxt1, -rv1b); accs(&WB, P->rbxt2, -rv2b);
        accs(&Pb->raxt1, wa1, rv1b); accs(&Pb->raxt2, wa1, rv2b);
        accs(&Pb->rbxt1, wb1, -rv1b); accs(&Pb->rbxt2, wb1, -rv2b);
    } else {
        l1b = lamb[1];
        l2b = lamb[2];
    }
    /* (7) normal impulse application */
    double dnb = 0.0;
    if (dynA) {
        dnb += P->ma * dot(r->n, VA) + P->iA * dot(P->raxn, WA);
        addInvMass(M, r->a, dn * dot(r->n, VA));
        addInvI(M, r->a, dn * dot(P->raxn, WA));
        accs(&Pb->raxn, WA, P->iA * dn);
    }
    if (dynB) {
        dnb -= P->mb * dot(r->n, VB) + P->iB * dot(P->rbxn, WB);
        addInvMass(M, r->b, -dn * dot(r->n, VB));
        addInvI(M, r->b, -dn * dot(P->rbxn, WB));
        accs(&Pb->rbxn, WB, -P->iB * dn);
    }
    /* (6) */
    lnpb += dnb;
    double lnb = -dnb;
    /* (5), (4) */
    double sb = (bits & BR_CLAMP) ? lnpb : 0.0;
    lnb += sb;
    double jnb = sb;
    /* (3) */
    double targetb = jnb / P->kN;
    double vnb = -jnb / P->kN;
    Pb->kN += -jnb * jn / P->kN;
    /* (2) */
    if (bits & BR_RESMAX) *vn0b += -r->e * targetb;
    else Pb->target0 += targetb;
    /* (1) */
    accs(&VA, r->n, vnb); accs(&WA, P->raxn, vnb);
    accs(&VB, r->n, -vnb); accs(&WB, P->rbxn, -vnb);
    accs(&Pb->raxn, wa, vnb); accs(&Pb->rbxn, wb, -vnb);
    *vbA = VA; *wbA = WA; *vbB = VB; *wbB = WB;
    lamb[0] = lnb; lamb[1] = l1b; lamb[2] = l2b;
}

/* warmStartContact on prepared arms (linear impulses only: rolling and
 * spinning impulses are zero in the model) */
static int warmActive(const double* lam) { return !(lam[0] <= 0.0 && lam[1] == 0.0 && lam[2] == 0.0); }

static void warmForward(const Mass* M, St* S, const Row* r, const Prep* P, const double* lam, int active) {
    if (!active) return;
    D3 imp = add(add(mul(r->n, lam[0]), mul(r->t1, lam[1])), mul(r->t2, lam[2]));
    applyImpulse(&S[r->a], &S[r->b], P, imp, cross(P->ra, imp), cross(P->rb, imp), M->prop[r->a].dyn,
                 M->prop[r->b].dyn);
}

static void warmReverse(const Mass* M, const Row* r, const Prep* P, const double* lam, D3* vbA, D3* wbA, D3* vbB,
                        D3* wbB, double* lamb, PrepBar* Pb, int active) {
    if (!active) return;
    D3 imp = add(add(mul(r->n, lam[0]), mul(r->t1, lam[1])), mul(r->t2, lam[2]));
    D3 ib = d3(0, 0, 0);
    if (M->prop[r->a].dyn) {
        accs(&ib, *vbA, P->ma);
        accs(&ib, cross(*wbA, P->ra), P->iA);
        accs(&Pb->ra, cross(imp, *wbA), P->iA);
        addInvMass(M, r->a, dot(imp, *vbA));
        addInvI(M, r->a, dot(cross(P->ra, imp), *wbA));
    }
    if (M->prop[r->b].dyn) {
        accs(&ib, *vbB, -P->mb);
        accs(&ib, cross(*wbB, P->rb), -P->iB);
        accs(&Pb->rb, cross(imp, *wbB), -P->iB);
        addInvMass(M, r->b, -dot(imp, *vbB));
        addInvI(M, r->b, -dot(cross(P->rb, imp), *wbB));
    }
    lamb[0] += dot(r->n, ib);
    lamb[1] += dot(r->t1, ib);
    lamb[2] += dot(r->t2, ib);
}

/* ---- the model ---------------------------------------------------------------- */

typedef struct {
    int n, steps, maxColor;
    const adjref_config* cfg;
    const Prop* prop;
    Mass M;
    /* per step */
    const uint32_t* stepStart;
    Row* rows;       /* all steps' rows */
    int32_t* src;    /* warm-start source (global row index of the previous step) or -1 */
    int32_t* vsrc;   /* vn0 source or -1 */
    double* lamRec;  /* recorded warm-start impulses (3 per row), used where no source applies */
    double* lamFin;  /* final impulses (3 per row) */
    double* vn0;     /* vn0 per row */
    int* order;      /* per step: rows in colour-major order (global indices) */
    /* branch hash */
    uint64_t hash;
} Model;

static void hashIn(Model* m, uint64_t v) {
    m->hash ^= v + 0x9e3779b97f4a7c15ull + (m->hash << 6) + (m->hash >> 2);
}

static void integrateVelocity(const Model* m, St* S, double h) {
    for (int i = 0; i < m->n; ++i) {
        const Prop* p = &m->prop[i];
        if (!p->dyn || p->locked || p->asleep) continue;
        S[i].v = add(S[i].v, mul(d3(m->cfg->gx, m->cfg->gy, m->cfg->gz), p->gs * h));
        S[i].v = mul(S[i].v, 1.0 / (1.0 + p->ld * h));
        S[i].w = mul(S[i].w, 1.0 / (1.0 + p->ad * h));
    }
}

static void integrateVelocityRev(const Model* m, D3* vb, D3* wb, double h) {
    for (int i = 0; i < m->n; ++i) {
        const Prop* p = &m->prop[i];
        if (!p->dyn || p->locked || p->asleep) continue;
        vb[i] = mul(vb[i], 1.0 / (1.0 + p->ld * h));
        wb[i] = mul(wb[i], 1.0 / (1.0 + p->ad * h));
    }
}

static int moves(const Prop* p) { return !p->stat && !p->locked && !p->asleep; }

static double rowVn0Own(const Model* m, const St* S, const Row* r) {
    D3 ra = anchorArm(&m->prop[r->a], S[r->a].q, r->la);
    D3 rb = anchorArm(&m->prop[r->b], S[r->b].q, r->lb);
    return dot(r->n, sub(S[r->a].v, S[r->b].v)) + dot(cross(ra, r->n), S[r->a].w) - dot(cross(rb, r->n), S[r->b].w);
}

/* Branch decisions to follow instead of deciding (adjref_force_branches):
 * per step, blocks of g_forcedRows bytes indexed by the step's row: per
 * substep the live gap's sign, the warm start's activity, per substep and
 * sweep the row bits (BR_*), per position pass the push's activity. */
static const uint8_t* g_forced = NULL;
static uint32_t g_forcedRows = 0;
/* The same layout, written with the decisions a run takes (adjref_record_branches). */
static uint8_t* g_record = NULL;
static uint32_t g_recordRows = 0;

static size_t branchBlocks(const adjref_config* c) {
    return (size_t)c->substeps * (1 + c->sweeps) + 1 + (size_t)c->positionIterations;
}

static const uint8_t* forcedStep(const Model* m, int t) {
    if (!g_forced) return NULL;
    return g_forced + (size_t)t * branchBlocks(m->cfg) * g_forcedRows;
}

/* block `block`, row k of step t in the recording (NULL when not recording) */
static uint8_t* recordAt(const Model* m, int t, size_t block, int k) {
    if (!g_record) return NULL;
    return g_record + ((size_t)t * branchBlocks(m->cfg) + block) * g_recordRows + (k - (int)m->stepStart[t]);
}

/* prep with the live gap's branch taken from the forced decisions */
static void prepAt(const Model* m, const St* S, int t, int sub, int k, double h, Prep* P) {
    prep(&m->M, S, &m->rows[k], h, P);
    const uint8_t* f = forcedStep(m, t);
    if (f) {
        P->gpos = f[(size_t)sub * g_forcedRows + (k - (int)m->stepStart[t])] != 0;
        P->target0 = P->gpos ? -P->gap / h : 0.0;
    }
    uint8_t* rec = recordAt(m, t, (size_t)sub, k);
    if (rec) *rec = (uint8_t)P->gpos;
}

static int warmAt(const Model* m, int t, int k, const double* lam) {
    const uint8_t* f = forcedStep(m, t);
    const int active = f ? f[(size_t)m->cfg->substeps * g_forcedRows + (k - (int)m->stepStart[t])] != 0
                         : warmActive(lam);
    uint8_t* rec = recordAt(m, t, (size_t)m->cfg->substeps, k);
    if (rec) *rec = (uint8_t)active;
    return active;
}

static int rowForcedAt(const Model* m, int t, int sub, int sweep, int k) {
    const uint8_t* f = forcedStep(m, t);
    if (!f) return -1;
    const size_t R = g_forcedRows, base = ((size_t)m->cfg->substeps + 1) * R;
    return f[base + ((size_t)sub * m->cfg->sweeps + sweep) * R + (k - (int)m->stepStart[t])];
}

static int pushForcedAt(const Model* m, int t, int it, int k) {
    const uint8_t* f = forcedStep(m, t);
    if (!f) return -1;
    const size_t R = g_forcedRows, base = ((size_t)m->cfg->substeps * (1 + m->cfg->sweeps) + 1) * R;
    return f[base + (size_t)it * R + (k - (int)m->stepStart[t])];
}

/* Relative perturbation of every state component after each substep
 * (adjref_set_state_noise): a deterministic function of (seed, step,
 * substep, body, component), so repeated evaluations see the same run. It
 * stands for an FP32 evaluation's per-substep rounding when estimating how
 * far the problem's conditioning lets an FP32 gradient sit from this one. */
static double g_noise = 0.0;
static uint64_t g_noiseSeed = 0;

static double noiseAt(int t, int s, int i, int c) {
    uint64_t x = g_noiseSeed ^ ((uint64_t)t << 40) ^ ((uint64_t)s << 32) ^ ((uint64_t)i << 8) ^ (uint64_t)c;
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33;
    return ((double)(x >> 11) / 9007199254740992.0 * 2.0 - 1.0) * g_noise;
}

static void perturbState(St* S, int t, int s, int i) {
    S->p.x *= 1.0 + noiseAt(t, s, i, 0); S->p.y *= 1.0 + noiseAt(t, s, i, 1); S->p.z *= 1.0 + noiseAt(t, s, i, 2);
    S->q.x *= 1.0 + noiseAt(t, s, i, 3); S->q.y *= 1.0 + noiseAt(t, s, i, 4);
    S->q.z *= 1.0 + noiseAt(t, s, i, 5); S->q.w *= 1.0 + noiseAt(t, s, i, 6);
    S->v.x *= 1.0 + noiseAt(t, s, i, 7); S->v.y *= 1.0 + noiseAt(t, s, i, 8); S->v.z *= 1.0 + noiseAt(t, s, i, 9);
    S->w.x *= 1.0 + noiseAt(t, s, i, 10); S->w.y *= 1.0 + noiseAt(t, s, i, 11);
    S->w.z *= 1.0 + noiseAt(t, s, i, 12);
}

/* tape of one step */
typedef struct {
    St* start;      /* state at step start (n) */
    St* sub;        /* per substep: state at substep start after velocity integration (n each) */
    St* end;        /* per substep: state after the sweeps, before transform integration (n each) */
    RowIn* rin;     /* per substep, sweep, colour-order row */
    St* corr;       /* state before the position correction (n) */
    double* push;   /* per pass, colour-order row: push (0 when inactive) */
    int* pact;      /* per pass, row: active */
    double* lamInit;
} Tape;

static void stepForward(Model* m, St* S, int t, Tape* T) {
    const adjref_config* cfg = m->cfg;
    const int S_ = cfg->substeps, W = cfg->sweeps;
    const double h = cfg->dt / S_;
    const int r0 = (int)m->stepStart[t], r1 = (int)m->stepStart[t + 1], R = r1 - r0;
    const int* ord = m->order + r0;
    if (T) memcpy(T->start, S, sizeof(St) * m->n);
    for (int i = 0; i < m->n; ++i) S[i].q = qnormalize(S[i].q, NULL);
    integrateVelocity(m, S, h);
    /* impulses and restitution references */
    double* lam = m->lamFin;  /* rows of this step accumulate in place */
    for (int k = r0; k < r1; ++k) {
        const int s = m->src[k];
        const double* from = (t > 0 && s >= 0) ? m->lamFin + 3 * s : m->lamRec + 3 * k;
        lam[3 * k] = from[0]; lam[3 * k + 1] = from[1]; lam[3 * k + 2] = from[2];
        if (T) memcpy(T->lamInit + 3 * (k - r0), from, sizeof(double) * 3);
        const int vs = m->vsrc[k];
        m->vn0[k] = vs < 0 ? rowVn0Own(m, S, &m->rows[k]) : t > 0 ? m->vn0[vs] : m->rows[k].vn0;
    }
    Prep* P = (Prep*)malloc(sizeof(Prep) * (R ? R : 1));
    for (int s = 0; s < S_; ++s) {
        if (s > 0) integrateVelocity(m, S, h);
        if (T) memcpy(T->sub + (size_t)s * m->n, S, sizeof(St) * m->n);
        for (int j = 0; j < R; ++j) {
            prepAt(m, S, t, s, ord[j], h, &P[j]);
            hashIn(m, (uint64_t)P[j].gpos);
        }
        if (s == 0)
            for (int j = 0; j < R; ++j) {
                const Row* r = &m->rows[ord[j]];
                const int active = warmAt(m, t, ord[j], lam + 3 * ord[j]);
                if (r->solved) warmForward(&m->M, S, r, &P[j], lam + 3 * ord[j], active);
                hashIn(m, (uint64_t)active);
            }
        for (int w = 0; w < W; ++w)
            for (int j = 0; j < R; ++j) {
                const int k = ord[j];
                const Row* r = &m->rows[k];
                RowIn* tin = T ? &T->rin[((size_t)s * W + w) * R + j] : NULL;
                if (!r->solved) { if (tin) tin->bits = BR_SKIP; continue; }
                RowIn tmp;
                rowForward(&m->M, S, r, &P[j], m->vn0[k], lam + 3 * k, tin ? tin : &tmp, rowForcedAt(m, t, s, w, k));
                uint8_t* rec = recordAt(m, t, (size_t)S_ + 1 + (size_t)s * W + w, k);
                if (rec) *rec = (uint8_t)(tin ? tin->bits : tmp.bits);
                hashIn(m, (uint64_t)(tin ? tin->bits : tmp.bits));
            }
        if (T) memcpy(T->end + (size_t)s * m->n, S, sizeof(St) * m->n);
        for (int i = 0; i < m->n; ++i) {
            if (!moves(&m->prop[i])) continue;
            S[i].p = add(S[i].p, mul(S[i].v, h));
            if (!m->prop[i].rotLocked) S[i].q = qintegrate(S[i].q, S[i].w, h);
            else S[i].w = d3(0, 0, 0);
            if (g_noise > 0.0) perturbState(&S[i], t, s, i);
        }
    }
    if (T) memcpy(T->corr, S, sizeof(St) * m->n);
    for (int it = 0; it < cfg->positionIterations; ++it)
        for (int j = 0; j < R; ++j) {
            const Row* r = &m->rows[ord[j]];
            double push = 0.0;
            int active = 0;
            const double ma = solverInvMass(&m->M, r->a), mb = solverInvMass(&m->M, r->b);
            if (r->solved && ma + mb > 0.0) {
                D3 ra = anchorArm(&m->prop[r->a], S[r->a].q, r->la);
                D3 rb = anchorArm(&m->prop[r->b], S[r->b].q, r->lb);
                double g = r->bias0 + dot(r->n, sub(add(S[r->a].p, ra), add(S[r->b].p, rb)));
                const int forced = pushForcedAt(m, t, it, ord[j]);
                if (forced >= 0 ? forced != 0 : g < -1e-3) {
                    double resolve = 0.6;
                    if (cfg->stackStabilization) {
                        D3 rv = sub(S[r->a].v, S[r->b].v);
                        if (dot(rv, rv) < 1e-4)
                            resolve += 0.2 * (cfg->stackStiffness / 1000.0) / (1.0 + cfg->stackDamping * h);
                    }
                    push = -resolve * (g + 1e-3) / (ma + mb);
                    active = 1;
                    if (m->prop[r->a].dyn && !m->prop[r->a].asleep) accs(&S[r->a].p, r->n, push * ma);
                    if (m->prop[r->b].dyn && !m->prop[r->b].asleep) accs(&S[r->b].p, r->n, -push * mb);
                }
            }
            hashIn(m, (uint64_t)active);
            uint8_t* rec = recordAt(m, t, (size_t)S_ * (1 + W) + 1 + (size_t)it, ord[j]);
            if (rec) *rec = (uint8_t)active;
            if (T) { T->push[(size_t)it * R + j] = push; T->pact[(size_t)it * R + j] = active; }
        }
    free(P);
}

/* Reverse of stepForward. sb: state adjoints after the step (updated to the
 * step start); lamb: adjoints of this step's final impulses (3 per row,
 * global index; updated: the previous step's rows receive their shares);
 * vn0b: adjoints of vn0 per row (same convention). */
static void stepReverse(Model* m, int t, Tape* T, D3* pb, D4* qb, D3* vb, D3* wb, double* lamb, double* vn0b) {
    const adjref_config* cfg = m->cfg;
    const int S_ = cfg->substeps, W = cfg->sweeps, n = m->n;
    const double h = cfg->dt / S_;
    const int r0 = (int)m->stepStart[t], r1 = (int)m->stepStart[t + 1], R = r1 - r0;
    const int* ord = m->order + r0;
    /* position correction */
    for (int it = cfg->positionIterations - 1; it >= 0; --it)
        for (int j = R - 1; j >= 0; --j) {
            if (!T->pact[(size_t)it * R + j]) continue;
            const Row* r = &m->rows[ord[j]];
            const double push = T->push[(size_t)it * R + j];
            const double ma = solverInvMass(&m->M, r->a), mb = solverInvMass(&m->M, r->b);
            double pushb = 0.0;
            if (m->prop[r->a].dyn && !m->prop[r->a].asleep) {
                pushb += ma * dot(r->n, pb[r->a]);
                addInvMass(&m->M, r->a, push * dot(r->n, pb[r->a]));
            }
            if (m->prop[r->b].dyn && !m->prop[r->b].asleep) {
                pushb -= mb * dot(r->n, pb[r->b]);
                addInvMass(&m->M, r->b, -push * dot(r->n, pb[r->b]));
            }
            /* push = -resolve (g + slop) / (ma + mb) */
            const double sum = ma + mb;
            double gb = 0.0;
            {
                /* d push / d g = -resolve / sum ; d push / d sum = -push / sum */
                double resolveOnly = 0.6;
                if (cfg->stackStabilization) {
                    D3 rv = sub(T->corr[r->a].v, T->corr[r->b].v);
                    if (dot(rv, rv) < 1e-4)
                        resolveOnly += 0.2 * (cfg->stackStiffness / 1000.0) / (1.0 + cfg->stackDamping * h);
                }
                gb = -resolveOnly / sum * pushb;
                double sumb = -push / sum * pushb;
                addInvMass(&m->M, r->a, sumb);
                addInvMass(&m->M, r->b, sumb);
            }
            /* g = bias0 + n . (pa + ra - pb - rb), orientations are the final ones */
            accs(&pb[r->a], r->n, gb);
            accs(&pb[r->b], r->n, -gb);
            if (!m->prop[r->a].sphere) rotRev(T->corr[r->a].q, r->la, mul(r->n, gb), &qb[r->a], NULL);
            if (!m->prop[r->b].sphere) rotRev(T->corr[r->b].q, r->lb, mul(r->n, -gb), &qb[r->b], NULL);
        }
    Prep* P = (Prep*)malloc(sizeof(Prep) * (R ? R : 1));
    PrepBar* Pb = (PrepBar*)malloc(sizeof(PrepBar) * (R ? R : 1));
    double* rvn0b = (double*)calloc(R ? R : 1, sizeof(double));
    for (int s = S_ - 1; s >= 0; --s) {
        const St* Ss = T->sub + (size_t)s * n;
        const St* Se = T->end + (size_t)s * n;
        /* transform integration */
        for (int i = 0; i < n; ++i) {
            if (!moves(&m->prop[i])) continue;
            if (!m->prop[i].rotLocked) {
                D4 qo = qb[i];
                D4 qz = {0, 0, 0, 0};
                qb[i] = qz;
                qintegrateRev(Se[i].q, Se[i].w, h, qo, &qb[i], &wb[i]);
            } else {
                wb[i] = d3(0, 0, 0);
            }
            accs(&vb[i], pb[i], h);
        }
        memset(Pb, 0, sizeof(PrepBar) * (R ? R : 1));
        for (int j = 0; j < R; ++j) prepAt(m, Ss, t, s, ord[j], h, &P[j]);
        /* sweeps */
        for (int w = W - 1; w >= 0; --w)
            for (int j = R - 1; j >= 0; --j) {
                const int k = ord[j];
                const Row* r = &m->rows[k];
                const RowIn* in = &T->rin[((size_t)s * W + w) * R + j];
                if (!r->solved || (in->bits & BR_SKIP)) continue;
                rowReverse(&m->M, r, &P[j], m->vn0[k], in, &vb[r->a], &wb[r->a], &vb[r->b], &wb[r->b],
                           lamb + 3 * k, &Pb[j], &rvn0b[j]);
            }
        if (s == 0) {
            for (int j = R - 1; j >= 0; --j) {
                const int k = ord[j];
                const Row* r = &m->rows[k];
                if (r->solved)
                    warmReverse(&m->M, r, &P[j], T->lamInit + 3 * (k - r0), &vb[r->a], &wb[r->a], &vb[r->b],
                                &wb[r->b], lamb + 3 * k, &Pb[j], warmAt(m, t, k, T->lamInit + 3 * (k - r0)));
            }
            /* restitution references of this step: own detection or a source */
            for (int j = 0; j < R; ++j) {
                const int k = ord[j];
                const Row* r = &m->rows[k];
                const double g = rvn0b[j] + vn0b[k];
                if (g == 0.0 || !r->solved) continue;
                const int vs = m->vsrc[k];
                if (vs >= 0) {  /* carried: to its source, or a constant from before the recorded steps */
                    if (t > 0) vn0b[vs] += g;
                    continue;
                }
                /* vn0 = n.(va - vb) + (ra x n).wa - (rb x n).wb at detection (= Ss for s == 0) */
                accs(&vb[r->a], r->n, g);
                accs(&vb[r->b], r->n, -g);
                accs(&wb[r->a], P[j].raxn, g);
                accs(&wb[r->b], P[j].rbxn, -g);
                accs(&Pb[j].raxn, Ss[r->a].w, g);
                accs(&Pb[j].rbxn, Ss[r->b].w, -g);
            }
        }
        for (int j = 0; j < R; ++j) {
            const Row* r = &m->rows[ord[j]];
            if (r->solved) prepRev(&m->M, Ss, r, h, &P[j], &Pb[j], pb, qb);
        }
        integrateVelocityRev(m, vb, wb, h);  /* s > 0: this substep's; s == 0: the prepare's */
    }
    /* orientation normalisation at the step start */
    for (int i = 0; i < n; ++i) {
        qb[i] = qnormalizeRev(T->start[i].q, qb[i]);
    }
    /* impulses received from the previous step */
    for (int k = r0; k < r1; ++k) {
        const int s = m->src[k];
        if (t > 0 && s >= 0) {
            lamb[3 * s] += lamb[3 * k];
            lamb[3 * s + 1] += lamb[3 * k + 1];
            lamb[3 * s + 2] += lamb[3 * k + 2];
        }
    }
    free(P);
    free(Pb);
    free(rvn0b);
}

/* colour-major order of one step's rows (stable) */
static void buildOrder(Model* m) {
    for (int t = 0; t < m->steps; ++t) {
        const int r0 = (int)m->stepStart[t], r1 = (int)m->stepStart[t + 1];
        int maxc = 0;
        for (int k = r0; k < r1; ++k) if (m->rows[k].color > maxc) maxc = m->rows[k].color;
        int pos = r0;
        for (int c = 0; c <= maxc; ++c)
            for (int k = r0; k < r1; ++k)
                if (m->rows[k].color == c) m->order[pos++] = k;
        for (int k = r0; k < r1; ++k)
            if (m->rows[k].color < 0) m->order[pos++] = k;
    }
}

static void stToArr(const St* S, int n, double* out) {
    for (int i = 0; i < n; ++i) {
        double* o = out + 13 * i;
        o[0] = S[i].p.x; o[1] = S[i].p.y; o[2] = S[i].p.z;
        o[3] = S[i].q.x; o[4] = S[i].q.y; o[5] = S[i].q.z; o[6] = S[i].q.w;
        o[7] = S[i].v.x; o[8] = S[i].v.y; o[9] = S[i].v.z;
        o[10] = S[i].w.x; o[11] = S[i].w.y; o[12] = S[i].w.z;
    }
}

/*
 * Runs the model over `steps` steps from state0 (n x 13 doubles: p, q, v, w)
 * with inverse masses invMass[n] and isotropic inverse inertias invI[n].
 * contacts/stepStart/src/color: the frozen contacts of every step (src: two
 * entries per contact, the warm-start source and the vn0 source as indices
 * into the previous step's contacts, 0xffffffff = none). Writes the final
 * state; with `seed` (dL/d final state, n x 13) also writes dL/d state0,
 * dL/d invMass and dL/d invI. *branchHash receives a hash of every branch the
 * forward took (equal hashes: the same active sets). Returns 0, or -1 when a
 * body has anisotropic inverse inertia.
 */
int adjref_run(const adjref_config* cfg, const vx_body* bodies, uint32_t n, const double* state0,
               const double* invMass, const double* invI, const vx_contact* contacts, const uint32_t* stepStart,
               const uint32_t* src, const int32_t* color, uint32_t steps, double* stateOut, const double* seed,
               double* grad, double* gradInvMass, double* gradInvI, uint64_t* branchHash) {
    for (uint32_t i = 0; i < n; ++i) {
        const vx_body* b = &bodies[i];
        if (b->motionType == VX_MOTION_DYNAMIC &&
            (b->invInertia.x != b->invInertia.y || b->invInertia.y != b->invInertia.z))
            return -1;
    }
    Model m;
    memset(&m, 0, sizeof(m));
    m.n = (int)n;
    m.steps = (int)steps;
    m.cfg = cfg;
    Prop* prop = (Prop*)malloc(sizeof(Prop) * n);
    for (uint32_t i = 0; i < n; ++i) prop[i] = propOf(&bodies[i]);
    m.prop = prop;
    double* gIm = (double*)calloc(n, sizeof(double));
    double* gIi = (double*)calloc(n, sizeof(double));
    m.M.prop = prop; m.M.invMass = invMass; m.M.invI = invI; m.M.gInvMass = gIm; m.M.gInvI = gIi;
    const uint32_t total = stepStart[steps];
    m.stepStart = stepStart;
    m.rows = (Row*)malloc(sizeof(Row) * (total ? total : 1));
    m.src = (int32_t*)malloc(sizeof(int32_t) * (total ? total : 1));
    m.vsrc = (int32_t*)malloc(sizeof(int32_t) * (total ? total : 1));
    m.lamRec = (double*)malloc(sizeof(double) * 3 * (total ? total : 1));
    m.lamFin = (double*)calloc(3 * (total ? total : 1), sizeof(double));
    m.vn0 = (double*)calloc(total ? total : 1, sizeof(double));
    m.order = (int*)malloc(sizeof(int) * (total ? total : 1));
    for (uint32_t t = 0; t < steps; ++t)
        for (uint32_t k = stepStart[t]; k < stepStart[t + 1]; ++k) {
            const vx_contact* c = &contacts[k];
            Row* r = &m.rows[k];
            r->a = (int)c->a; r->b = (int)c->b;
            r->solved = !prop[c->a].sensor && !prop[c->b].sensor;
            r->n = fromf(c->normal);
            tangents(r->n, &r->t1, &r->t2);
            r->la = fromf(c->localAnchorA); r->lb = fromf(c->localAnchorB);
            r->bias0 = c->bias0; r->e = c->restitution; r->f1 = c->friction1; r->f2 = c->friction2;
            r->vn0 = c->vn0;
            r->color = color[k];
            const uint32_t prev0 = t > 0 ? stepStart[t - 1] : 0;
            m.src[k] = src[2 * k] == 0xffffffffu ? -1 : (int32_t)(prev0 + src[2 * k]);
            m.vsrc[k] = src[2 * k + 1] == 0xffffffffu ? -1 : (int32_t)(prev0 + src[2 * k + 1]);
            m.lamRec[3 * k] = c->normalImpulse; m.lamRec[3 * k + 1] = c->tangentImpulse1;
            m.lamRec[3 * k + 2] = c->tangentImpulse2;
        }
    buildOrder(&m);
    St* S = (St*)malloc(sizeof(St) * n);
    for (uint32_t i = 0; i < n; ++i) {
        const double* s = state0 + 13 * i;
        S[i].p = d3(s[0], s[1], s[2]);
        D4 q = {s[3], s[4], s[5], s[6]};
        S[i].q = q;
        S[i].v = d3(s[7], s[8], s[9]);
        S[i].w = d3(s[10], s[11], s[12]);
    }
    const int S_ = cfg->substeps, W = cfg->sweeps;
    Tape* tapes = NULL;
    if (seed) tapes = (Tape*)calloc(steps ? steps : 1, sizeof(Tape));
    for (uint32_t t = 0; t < steps; ++t) {
        Tape* T = NULL;
        if (seed) {
            const size_t R = stepStart[t + 1] - stepStart[t];
            T = &tapes[t];
            T->start = (St*)malloc(sizeof(St) * n);
            T->sub = (St*)malloc(sizeof(St) * n * S_);
            T->end = (St*)malloc(sizeof(St) * n * S_);
            T->rin = (RowIn*)malloc(sizeof(RowIn) * (R ? R : 1) * S_ * W);
            T->corr = (St*)malloc(sizeof(St) * n);
            T->push = (double*)malloc(sizeof(double) * (R ? R : 1) * (cfg->positionIterations + 1));
            T->pact = (int*)malloc(sizeof(int) * (R ? R : 1) * (cfg->positionIterations + 1));
            T->lamInit = (double*)malloc(sizeof(double) * 3 * (R ? R : 1));
        }
        stepForward(&m, S, (int)t, T);
    }
    stToArr(S, (int)n, stateOut);
    if (seed) {
        D3* pb = (D3*)calloc(n, sizeof(D3));
        D4* qb = (D4*)calloc(n, sizeof(D4));
        D3* vb = (D3*)calloc(n, sizeof(D3));
        D3* wb = (D3*)calloc(n, sizeof(D3));
        for (uint32_t i = 0; i < n; ++i) {
            const double* s = seed + 13 * i;
            pb[i] = d3(s[0], s[1], s[2]);
            qb[i].x = s[3]; qb[i].y = s[4]; qb[i].z = s[5]; qb[i].w = s[6];
            vb[i] = d3(s[7], s[8], s[9]);
            wb[i] = d3(s[10], s[11], s[12]);
        }
        double* lamb = (double*)calloc(3 * (total ? total : 1), sizeof(double));
        double* vn0b = (double*)calloc(total ? total : 1, sizeof(double));
        for (int t = (int)steps - 1; t >= 0; --t) stepReverse(&m, t, &tapes[t], pb, qb, vb, wb, lamb, vn0b);
        for (uint32_t i = 0; i < n; ++i) {
            double* g = grad + 13 * i;
            g[0] = pb[i].x; g[1] = pb[i].y; g[2] = pb[i].z;
            g[3] = qb[i].x; g[4] = qb[i].y; g[5] = qb[i].z; g[6] = qb[i].w;
            g[7] = vb[i].x; g[8] = vb[i].y; g[9] = vb[i].z;
            g[10] = wb[i].x; g[11] = wb[i].y; g[12] = wb[i].z;
            if (gradInvMass) gradInvMass[i] = gIm[i];
            if (gradInvI) gradInvI[i] = gIi[i];
        }
        free(pb); free(qb); free(vb); free(wb); free(lamb); free(vn0b);
        for (uint32_t t = 0; t < steps; ++t) {
            free(tapes[t].start); free(tapes[t].sub); free(tapes[t].end); free(tapes[t].rin);
            free(tapes[t].corr); free(tapes[t].push); free(tapes[t].pact); free(tapes[t].lamInit);
        }
        free(tapes);
    }
    if (branchHash) *branchHash = m.hash;
    free(S); free(prop); free(gIm); free(gIi); free(m.rows); free(m.src); free(m.vsrc); free(m.lamRec);
    free(m.lamFin); free(m.vn0); free(m.order);
    return 0;
}

/* Follow the given branch decisions (layout at g_forced; rows = bytes per
 * block) in the following adjref_run calls, instead of deciding them: the
 * derivative of the piece another run took. Null stops it. */
void adjref_force_branches(const uint8_t* bits, uint32_t rows) {
    g_forced = bits;
    g_forcedRows = rows;
}

/* Write the branch decisions of the following adjref_run calls to `out`
 * (the layout adjref_force_branches reads; rows = bytes per block, at least
 * the most rows of any step). Null stops it. */
void adjref_record_branches(uint8_t* out, uint32_t rows) {
    g_record = out;
    g_recordRows = rows;
}

/* Perturb the state by up to `relative` after every substep of the following
 * adjref_run calls (0 = off); `seed` picks the perturbation. */
void adjref_set_state_noise(double relative, uint64_t seed) {
    g_noise = relative;
    g_noiseSeed = seed;
}
