// Candidates of the unweighting: counter-based uniforms, the five-number phase-space map of
// massless 2 -> 3 at fixed sqrt(s) and the jet cuts, in f64 on the device.
//
// Candidate i of a stream with seed S: a xorshift64 stream (shifts 13, 7, 17; uniform =
// ((state >> 11) + 0.5) / 2^53) started at splitmix64(S ^ (i * 0xD1B54A32D192ED03)) | 1. Uniforms
// 0-4 are the phase-space numbers, 5 the first accept/reject number, 6 the second.
//
// The map (sequential two-body decays, each variable importance-sampled where |M|^2 peaks):
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
#pragma once
#include <stdint.h>

namespace pacuda {
namespace phase {

constexpr int UNIFORMS = 7;

struct Cuts {
    double pt_min, eta_max, dr_min;
};

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ void uniforms(uint64_t seed, uint64_t index, double (&u)[UNIFORMS]) {
    uint64_t state = splitmix64(seed ^ (index * 0xD1B54A32D192ED03ull)) | 1ull;
#pragma unroll
    for (int k = 0; k < UNIFORMS; k++) {
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

// the map's weight J from uniforms u[0..4] alone (no momenta)
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

// pT > pt_min, |eta| < eta_max and pairwise Delta R > dr_min on legs 2..4; the first two as
// pT^2 > pt_min^2 and |pz| < pT sinh(eta_max) (no transcendental function for a point they reject),
// eta = asinh(pz / pT) and phi = atan2(py, px) only for the Delta R of points that pass them
__device__ __forceinline__ bool passes(const double (&p)[5][4], const Cuts &c) {
    const double sh = sinh(c.eta_max);
    double pt[3];
    for (int i = 0; i < 3; i++) {
        const double *q = p[2 + i];
        const double pt2 = q[1] * q[1] + q[2] * q[2];
        if (!(pt2 > c.pt_min * c.pt_min)) return false;
        pt[i] = sqrt(pt2);
        if (!(fabs(q[3]) < pt[i] * sh)) return false;
    }
    double eta[3], phi[3];
    for (int i = 0; i < 3; i++) {
        eta[i] = asinh(p[2 + i][3] / pt[i]);
        phi[i] = atan2(p[2 + i][2], p[2 + i][1]);
    }
    const double pi = 3.141592653589793;
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++) {
            double d = fabs(phi[i] - phi[j]);
            if (d > pi) d = 2.0 * pi - d;
            const double de = eta[i] - eta[j];
            if (!(de * de + d * d > c.dr_min * c.dr_min)) return false;
        }
    return true;
}

}  // namespace phase
}  // namespace pacuda
