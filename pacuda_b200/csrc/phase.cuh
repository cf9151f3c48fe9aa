// Candidates of the unweighting: counter-based uniforms, the phase-space maps of massless 2 -> 3
// (five numbers) and 2 -> 4 (eight numbers) at fixed sqrt(s) and the jet cuts, in f64 on the
// device.
//
// Candidate i of a stream with seed S: a xorshift64 stream (shifts 13, 7, 17; uniform =
// ((state >> 11) + 0.5) / 2^53) started at splitmix64(S ^ (i * 0xD1B54A32D192ED03)) | 1. For N
// final-state partons, uniforms 0 .. 3N - 5 are the phase-space numbers, 3N - 4 the first
// accept/reject number and 3N - 3 the second.
//
// The 2 -> 3 map (sequential two-body decays, each variable importance-sampled where |M|^2 peaks):
//   s23 = s sigma(y), y = L (2 x1 - 1), sigma(y) = 1 / (1 + e^-y): logarithmic towards both the
//     collinear 2 || 3 end (small s23) and the soft-p1 end (s23 near s);
//   p1 in the centre-of-mass frame with |p1| = (s - s23) / (2 sqrt(s)), cos(theta1) =
//     tanh(E1 (2 x2 - 1)) (flat in p1's pseudorapidity: the beam-collinear peaks), phi1 = 2 pi x3;
//   p2 and p3 back to back in the rest frame of q = P - p1 with |p| = sqrt(s23) / 2, cos(theta2) =
//     tanh(E2 (2 x4 - 1)), phi2 = 2 pi x5, boosted along q.
// Its weight, the phase-space density of the unit cube:
//   J = s (1 - sigma) / (128 pi^3) x 2 L sigma (1 - sigma) x E1 (1 - cos^2 theta1) x E2 (1 - cos^2 theta2),
// the flat map's s (1 - x1) / (128 pi^3) times the three variables' Jacobians. With L = 16 the map
// reaches m23 down to 4.4 GeV at 13 TeV (the cuts need at least 8 GeV); E1 = 5.5 covers every p1
// inside |eta| < 5; E2 = 7 leaves out a q-frame solid angle of 1.7e-6 around the z axis.
// Legs: 0, 1 the beams (sqrt(s)/2)(1, 0, 0, +-1), 2 = p1, 3 = p2, 4 = p3.
//
// The 2 -> 4 map adds one decay: P -> p1 + Q, Q -> p2 + R, R -> p3 + p4 with
//   s_Q = s sigma(L (2 x1 - 1)), s_R = s_Q sigma(L (2 x4 - 1));
//   p1 as above (x2, x3), |p1| = (s - s_Q) / (2 sqrt(s));
//   p2 in the rest frame of Q, |p2| = (s_Q - s_R) / (2 sqrt(s_Q)), cos(theta2) = tanh(E2 (2 x5 - 1)),
//     phi2 = 2 pi x6, R opposite;
//   p3, p4 back to back in the rest frame of R, |p| = sqrt(s_R) / 2, cos(theta3) = tanh(E2 (2 x7 - 1)),
//     phi3 = 2 pi x8; boosted to Q's frame along R, then with p2 to the lab along Q;
// from dPhi_4 = dPhi_2(P; p1, Q) ds_Q / 2 pi dPhi_2(Q; p2, R) ds_R / 2 pi dPhi_2(R; p3, p4) and
// dPhi_2(K; k1 massless, k2 of mass^2 m) = (K^2 - m) / (32 pi^2 K^2) dOmega:
//   J = s s_Q (1 - sigma1) (1 - sigma2) / (2048 pi^5) x 2 L sigma1 (1 - sigma1) x 2 L sigma2 (1 - sigma2)
//       x E1 (1 - c1^2) x E2 (1 - c2^2) x E2 (1 - c3^2)
// (flat variables integrate it to the massless four-body volume s^2 / (24576 pi^5)).
// Legs: 0, 1 the beams, 2 = p1, 3 = p2, 4 = p3, 5 = p4.
#pragma once
#include <stdint.h>

namespace pacuda {
namespace phase {

// N final-state partons: 3N - 2 uniforms, 3N - 4 of them phase-space numbers, N + 2 legs
template <int N> struct Space {
    static constexpr int UNIFORMS = 3 * N - 2, NUMBERS = 3 * N - 4, LEGS = N + 2;
};
constexpr int UNIFORMS = Space<3>::UNIFORMS;
constexpr int MAX_UNIFORMS = Space<4>::UNIFORMS;

struct Cuts {
    double pt_min, eta_max, dr_min;
};

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <int U> __device__ __forceinline__ void uniforms(uint64_t seed, uint64_t index, double (&u)[U]) {
    uint64_t state = splitmix64(seed ^ (index * 0xD1B54A32D192ED03ull)) | 1ull;
#pragma unroll
    for (int k = 0; k < U; k++) {
        state ^= state << 13;
        state ^= state >> 7;
        state ^= state << 17;
        u[k] = ((double)(state >> 11) + 0.5) / 9007199254740992.0;
    }
}

// p (rest frame of q) boosted by the velocity b of q
__device__ __forceinline__ void boost(const double (&p)[4], const double (&b)[3], double (&out)[4]) {
    const double b2 = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
    const double g = 1.0 / sqrt(1.0 - b2);
    const double bp = b[0] * p[1] + b[1] * p[2] + b[2] * p[3];
    const double gg = b2 > 0.0 ? (g - 1.0) / b2 : 0.0;
    out[0] = g * (p[0] + bp);
    const double f = gg * bp + g * p[0];
    out[1] = p[1] + f * b[0];
    out[2] = p[2] + f * b[1];
    out[3] = p[3] + f * b[2];
}

constexpr double MAP_L = 16.0, MAP_E1 = 5.5, MAP_E2 = 7.0;

// the 2 -> 3 map's weight J from uniforms u[0..4] alone (no momenta)
__device__ __forceinline__ double weight(const double (&u)[UNIFORMS], double sqrt_s) {
    const double s = sqrt_s * sqrt_s, pi = 3.141592653589793;
    const double sg = 1.0 / (1.0 + exp(-MAP_L * (2.0 * u[0] - 1.0)));
    const double c1 = tanh(MAP_E1 * (2.0 * u[1] - 1.0)), c2 = tanh(MAP_E2 * (2.0 * u[3] - 1.0));
    return s * (1.0 - sg) / (128.0 * pi * pi * pi) * (2.0 * MAP_L * sg * (1.0 - sg)) * (MAP_E1 * (1.0 - c1 * c1)) *
           (MAP_E2 * (1.0 - c2 * c2));
}

// the five legs' momenta [leg][E, px, py, pz] and the weight J of uniforms u[0..4]
__device__ __forceinline__ double map(const double (&u)[UNIFORMS], double sqrt_s, double (&p)[5][4]) {
    const double s = sqrt_s * sqrt_s, pi = 3.141592653589793;
    const double sg = 1.0 / (1.0 + exp(-MAP_L * (2.0 * u[0] - 1.0)));
    const double s23 = s * sg;
    const double e1 = (s - s23) / (2.0 * sqrt_s);
    const double c1 = tanh(MAP_E1 * (2.0 * u[1] - 1.0)), st1 = sqrt(fmax(0.0, 1.0 - c1 * c1)), f1 = 2.0 * pi * u[2];
    double sf1, cf1;
    sincos(f1, &sf1, &cf1);
    p[0][0] = 0.5 * sqrt_s; p[0][1] = 0.0; p[0][2] = 0.0; p[0][3] = 0.5 * sqrt_s;
    p[1][0] = 0.5 * sqrt_s; p[1][1] = 0.0; p[1][2] = 0.0; p[1][3] = -0.5 * sqrt_s;
    p[2][0] = e1; p[2][1] = e1 * st1 * cf1; p[2][2] = e1 * st1 * sf1; p[2][3] = e1 * c1;
    const double k = 0.5 * sqrt(s23);
    const double c2 = tanh(MAP_E2 * (2.0 * u[3] - 1.0)), st2 = sqrt(fmax(0.0, 1.0 - c2 * c2)), f2 = 2.0 * pi * u[4];
    double sf2, cf2;
    sincos(f2, &sf2, &cf2);
    const double r2[4] = {k, k * st2 * cf2, k * st2 * sf2, k * c2};
    const double r3[4] = {k, -r2[1], -r2[2], -r2[3]};
    const double eq = sqrt_s - e1;
    const double b[3] = {-p[2][1] / eq, -p[2][2] / eq, -p[2][3] / eq};
    double o[4];
    boost(r2, b, o);
    for (int c = 0; c < 4; c++) p[3][c] = o[c];
    boost(r3, b, o);
    for (int c = 0; c < 4; c++) p[4][c] = o[c];
    return s * (1.0 - sg) / (128.0 * pi * pi * pi) * (2.0 * MAP_L * sg * (1.0 - sg)) * (MAP_E1 * (1.0 - c1 * c1)) *
           (MAP_E2 * (1.0 - c2 * c2));
}

// the 2 -> 4 map: the six legs' momenta [leg][E, px, py, pz] and the weight J of uniforms u[0..7]
__device__ __forceinline__ double map4(const double (&u)[Space<4>::UNIFORMS], double sqrt_s, double (&p)[6][4]) {
    const double s = sqrt_s * sqrt_s, pi = 3.141592653589793;
    const double sg1 = 1.0 / (1.0 + exp(-MAP_L * (2.0 * u[0] - 1.0)));
    const double sq = s * sg1;
    const double sg2 = 1.0 / (1.0 + exp(-MAP_L * (2.0 * u[3] - 1.0)));
    const double sr = sq * sg2;
    // p1 in the centre-of-mass frame
    const double e1 = (s - sq) / (2.0 * sqrt_s);
    const double c1 = tanh(MAP_E1 * (2.0 * u[1] - 1.0)), st1 = sqrt(fmax(0.0, 1.0 - c1 * c1)), f1 = 2.0 * pi * u[2];
    double sf1, cf1;
    sincos(f1, &sf1, &cf1);
    p[0][0] = 0.5 * sqrt_s; p[0][1] = 0.0; p[0][2] = 0.0; p[0][3] = 0.5 * sqrt_s;
    p[1][0] = 0.5 * sqrt_s; p[1][1] = 0.0; p[1][2] = 0.0; p[1][3] = -0.5 * sqrt_s;
    p[2][0] = e1; p[2][1] = e1 * st1 * cf1; p[2][2] = e1 * st1 * sf1; p[2][3] = e1 * c1;
    // p2 and R in the rest frame of Q
    const double mq = sqrt(sq);
    const double k2 = (sq - sr) / (2.0 * mq);
    const double c2 = tanh(MAP_E2 * (2.0 * u[4] - 1.0)), st2 = sqrt(fmax(0.0, 1.0 - c2 * c2)), f2 = 2.0 * pi * u[5];
    double sf2, cf2;
    sincos(f2, &sf2, &cf2);
    const double q2[4] = {k2, k2 * st2 * cf2, k2 * st2 * sf2, k2 * c2};
    const double er = (sq + sr) / (2.0 * mq);
    // p3 and p4 back to back in the rest frame of R, then into Q's frame along R (velocity -q2 / er)
    const double k3 = 0.5 * sqrt(sr);
    const double c3 = tanh(MAP_E2 * (2.0 * u[6] - 1.0)), st3 = sqrt(fmax(0.0, 1.0 - c3 * c3)), f3 = 2.0 * pi * u[7];
    double sf3, cf3;
    sincos(f3, &sf3, &cf3);
    const double r3[4] = {k3, k3 * st3 * cf3, k3 * st3 * sf3, k3 * c3};
    const double r4[4] = {k3, -r3[1], -r3[2], -r3[3]};
    const double br[3] = {-q2[1] / er, -q2[2] / er, -q2[3] / er};
    double q3[4], q4[4];
    boost(r3, br, q3);
    boost(r4, br, q4);
    // everything in Q's frame to the lab along Q (velocity -p1 / (sqrt(s) - e1))
    const double eq = sqrt_s - e1;
    const double bq[3] = {-p[2][1] / eq, -p[2][2] / eq, -p[2][3] / eq};
    double o[4];
    boost(q2, bq, o);
    for (int c = 0; c < 4; c++) p[3][c] = o[c];
    boost(q3, bq, o);
    for (int c = 0; c < 4; c++) p[4][c] = o[c];
    boost(q4, bq, o);
    for (int c = 0; c < 4; c++) p[5][c] = o[c];
    return s * sq * (1.0 - sg1) * (1.0 - sg2) / (2048.0 * pi * pi * pi * pi * pi) * (2.0 * MAP_L * sg1 * (1.0 - sg1)) *
           (2.0 * MAP_L * sg2 * (1.0 - sg2)) * (MAP_E1 * (1.0 - c1 * c1)) * (MAP_E2 * (1.0 - c2 * c2)) *
           (MAP_E2 * (1.0 - c3 * c3));
}

// the map of N final-state partons (3 or 4)
template <int N> struct Map;
template <> struct Map<3> {
    __device__ __forceinline__ static double momenta(const double (&u)[Space<3>::UNIFORMS], double sqrt_s,
                                                     double (&p)[5][4]) {
        return map(u, sqrt_s, p);
    }
};
template <> struct Map<4> {
    __device__ __forceinline__ static double momenta(const double (&u)[Space<4>::UNIFORMS], double sqrt_s,
                                                     double (&p)[6][4]) {
        return map4(u, sqrt_s, p);
    }
};

// pT > pt_min, |eta| < eta_max and pairwise Delta R > dr_min on legs 2 .. L - 1; the first two as
// pT^2 > pt_min^2 and |pz| < pT sinh(eta_max) (no transcendental function for a point they reject),
// eta = asinh(pz / pT) and phi = atan2(py, px) only for the Delta R of points that pass them
template <int L> __device__ __forceinline__ bool passes(const double (&p)[L][4], const Cuts &c) {
    constexpr int F = L - 2;
    const double sh = sinh(c.eta_max);
    double pt[F];
    for (int i = 0; i < F; i++) {
        const double *q = p[2 + i];
        const double pt2 = q[1] * q[1] + q[2] * q[2];
        if (!(pt2 > c.pt_min * c.pt_min)) return false;
        pt[i] = sqrt(pt2);
        if (!(fabs(q[3]) < pt[i] * sh)) return false;
    }
    double eta[F], phi[F];
    for (int i = 0; i < F; i++) {
        eta[i] = asinh(p[2 + i][3] / pt[i]);
        phi[i] = atan2(p[2 + i][2], p[2 + i][1]);
    }
    const double pi = 3.141592653589793;
    for (int i = 0; i < F; i++)
        for (int j = i + 1; j < F; j++) {
            double d = fabs(phi[i] - phi[j]);
            if (d > pi) d = 2.0 * pi - d;
            const double de = eta[i] - eta[j];
            if (!(de * de + d * d > c.dr_min * c.dr_min)) return false;
        }
    return true;
}

// ---- a first look in f32: candidates that certainly fail the cuts ----------------------------
// The f64 map above defines every candidate's point, and the cuts on it decide the list. Most
// candidates fail by a wide margin (a soft or collinear parton), so the listing first maps each
// one in f32, written to stay accurate where the f64 form cancels: 1 - sigma, cos(theta) and
// sin(theta) from one exponential each, and a boost by velocity |q| / E_q of a frame of mass m
// with gamma - 1 = |q|^2 / (m (E_q + m)) and gamma beta = |q| / m instead of 1 / sqrt(1 - beta^2).
// Its uniforms are the same stream's states read to 24 bits, its exponentials and angles the
// hardware approximations (relative errors near 2^-21). Every final-state component it gives then
// differs from the f64 map's by about 5e-7 sqrt(s) at most (the 24-bit uniforms dominate; a float32
// restatement of these formulas on 4e5 candidates of each map stays below that against the f64
// map), 40 times less than the margin: a candidate is dropped here only when it fails a cut by more
// than PHASE32_DELTA = 2e-5 sqrt(s) per component allows (pT by 2 delta, |pz| - pT sinh(eta_max)
// by (1 + 1.5 sinh(eta_max)) delta, Delta R by the propagated bounds on eta and phi). Every other
// candidate goes through the f64 map and cuts, so the list is the f64 decision's.
constexpr float PHASE32_DELTA = 2e-5f;

// the first k uniforms of candidate `index` to 24 bits (the states of uniforms() above)
template <int K> __device__ __forceinline__ void uniforms32(uint64_t seed, uint64_t index, float (&u)[K]) {
    uint64_t state = splitmix64(seed ^ (index * 0xD1B54A32D192ED03ull)) | 1ull;
#pragma unroll
    for (int k = 0; k < K; k++) {
        state ^= state << 13;
        state ^= state >> 7;
        state ^= state << 17;
        u[k] = ((float)(uint32_t)(state >> 40) + 0.5f) * 5.9604644775390625e-8f;
    }
}

// cos(theta) = tanh(x), sin(theta) = 1 / cosh(x) from t = e^-|x|, and (cos, sin)(2 pi v): a unit
// direction
__device__ __forceinline__ void direction32(float x, float v, float (&n)[3]) {
    const float t = __expf(-fabsf(x)), t2 = t * t, r = 1.0f / (1.0f + t2);
    const float c = copysignf((1.0f - t2) * r, x), st = 2.0f * t * r;
    float sp, cp;
    __sincosf(3.14159265358979f * (2.0f * v - 1.0f), &sp, &cp);  // the angle 2 pi v - pi
    n[0] = -st * cp;
    n[1] = -st * sp;
    n[2] = c;
}

// the decay of a frame of mass m moving along the unit vector w with momentum q and energy e
// into two massless partons back to back along +-n in its rest frame: their momenta in the
// frame where it moves (its rest-frame momentum k = m / 2)
__device__ __forceinline__ void decay32(float m, float e, float q, const float (&w)[3], const float (&n)[3],
                                        float (&a)[3], float (&b)[3]) {
    const float k = 0.5f * m, cw = n[0] * w[0] + n[1] * w[1] + n[2] * w[2];
    const float along = q * q * cw / (2.0f * (e + m)), mid = 0.5f * q;
    for (int i = 0; i < 3; i++) {
        a[i] = k * n[i] + (along + mid) * w[i];
        b[i] = -k * n[i] + (mid - along) * w[i];
    }
}

// a momentum (energy en, vector v) in the frame of mass m moving along w with momentum q and
// energy e, seen where it moves: the vector part
__device__ __forceinline__ void boost32(float m, float e, float q, const float (&w)[3], float en, const float (&v)[3],
                                        float (&out)[3]) {
    const float par = v[0] * w[0] + v[1] * w[1] + v[2] * w[2];
    const float f = (q * q * par / (e + m) + q * en) / m;
    for (int i = 0; i < 3; i++) out[i] = v[i] + f * w[i];
}

// sigma(L (2 u - 1)) and 1 - sigma from one exponential
__device__ __forceinline__ void logistic32(float u, float &sg, float &omsg) {
    const float ey = __expf(-(float)MAP_L * (2.0f * u - 1.0f)), r = 1.0f / (1.0f + ey);
    sg = r;
    omsg = ey * r;
}

// the final-state partons' (px, py, pz) of the 2 -> 3 and 2 -> 4 maps in f32
__device__ __forceinline__ void final32(const float (&u)[Space<3>::NUMBERS], double sqrt_s, float (&p)[3][3]) {
    const float rs = (float)sqrt_s;
    float sg, omsg;
    logistic32(u[0], sg, omsg);
    const float e1 = 0.5f * rs * omsg, eq = 0.5f * rs * (1.0f + sg), mq = rs * sqrtf(sg);
    float n1[3], n2[3], w[3];
    direction32((float)MAP_E1 * (2.0f * u[1] - 1.0f), u[2], n1);
    for (int i = 0; i < 3; i++) {
        p[0][i] = e1 * n1[i];
        w[i] = -n1[i];
    }
    direction32((float)MAP_E2 * (2.0f * u[3] - 1.0f), u[4], n2);
    decay32(mq, eq, e1, w, n2, p[1], p[2]);
}

__device__ __forceinline__ void final32(const float (&u)[Space<4>::NUMBERS], double sqrt_s, float (&p)[4][3]) {
    const float rs = (float)sqrt_s;
    float sg1, omsg1, sg2, omsg2;
    logistic32(u[0], sg1, omsg1);
    logistic32(u[3], sg2, omsg2);
    const float e1 = 0.5f * rs * omsg1, eq = 0.5f * rs * (1.0f + sg1), mq = rs * sqrtf(sg1);
    const float k2 = 0.5f * mq * omsg2, er = 0.5f * mq * (1.0f + sg2), mr = mq * sqrtf(sg2);
    float n1[3], n2[3], n3[3], w[3], v[3];
    direction32((float)MAP_E1 * (2.0f * u[1] - 1.0f), u[2], n1);
    for (int i = 0; i < 3; i++) {
        p[0][i] = e1 * n1[i];
        w[i] = -n1[i];
    }
    direction32((float)MAP_E2 * (2.0f * u[4] - 1.0f), u[5], n2);
    direction32((float)MAP_E2 * (2.0f * u[6] - 1.0f), u[7], n3);
    // in Q's rest frame: p2 = k2 n2, R moving along -n2; p3, p4 from R's decay
    float q2[3], q3[3], q4[3];
    for (int i = 0; i < 3; i++) {
        q2[i] = k2 * n2[i];
        v[i] = -n2[i];
    }
    decay32(mr, er, k2, v, n3, q3, q4);
    const float c3 = n3[0] * v[0] + n3[1] * v[1] + n3[2] * v[2];
    const float en3 = 0.5f * (er + k2 * c3), en4 = 0.5f * (er - k2 * c3);
    // to the lab along Q
    boost32(mq, eq, e1, w, k2, q2, p[1]);
    boost32(mq, eq, e1, w, en3, q3, p[2]);
    boost32(mq, eq, e1, w, en4, q4, p[3]);
}

// whether the candidate whose f32 partons are p certainly fails the cuts (see above)
template <int F>
__device__ __forceinline__ bool surely_fails32(const float (&p)[F][3], double sqrt_s, const Cuts &c) {
    const float d = PHASE32_DELTA * (float)sqrt_s, sh = sinhf((float)c.eta_max);
    float pt[F];
    for (int i = 0; i < F; i++) {
        pt[i] = sqrtf(p[i][0] * p[i][0] + p[i][1] * p[i][1]);
        if (pt[i] < (float)c.pt_min - 2.0f * d) return true;
        if (fabsf(p[i][2]) - pt[i] * sh > d * (1.0f + 1.5f * sh)) return true;
    }
    float eta[F], phi[F], err[F];
    for (int i = 0; i < F; i++) {
        const float low = pt[i] - 2.0f * d;
        if (!(low > 0.0f)) return false;
        const float z = p[i][2] / pt[i];
        eta[i] = copysignf(__logf(fabsf(z) + sqrtf(z * z + 1.0f)), z);
        phi[i] = atan2f(p[i][1], p[i][0]);
        err[i] = 4.0f * d / low + 1e-5f;  // eta's bound 2.5 d / low, phi's 1.5 d / low, the functions' rounding
    }
    const float pi = 3.14159265f;
    for (int i = 0; i < F; i++)
        for (int j = i + 1; j < F; j++) {
            float dp = fabsf(phi[i] - phi[j]);
            if (dp > pi) dp = 2.0f * pi - dp;
            const float de = eta[i] - eta[j];
            if (sqrtf(de * de + dp * dp) + err[i] + err[j] + 1e-5f < (float)c.dr_min) return true;
        }
    return false;
}

}  // namespace phase
}  // namespace pacuda
