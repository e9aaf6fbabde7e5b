// sgfd_oracle.cpp — CPU ORACLE for the staggered-grid elastic timestep loop.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
// baseline legs of bench.py load this library, and only as the checker (or as
// the timed CPU baseline).  The product (libsgfd.so) never links or calls it.
//
// What it is: a plain C++ restatement, in FP32 or FP64, of the single-GPU PML
// program of the reference (3DGPUwithPML_1DArraySingleGPU_optimization/, "OPT/"
// below; identical kernels in 3DGPUwithPML_1DArraySingleGPU_concise/, "CON/").
// Parity pins (tests/test_oracle_golden.py, tests/test_ref_pin.py):
//   - the reference's shipped station trace CON/stationData.txt (1500 txx
//     samples of CON/main.cu's configuration, 6 significant digits);
//   - the reference OPT program itself, compiled from its own sources by
//     oracle/Makefile into oracle/_ref/ and run on a GPU, on homogeneous and
//     heterogeneous media (the only pin for the two index quirks below).
//
// The algorithm, per time step `it` (OPT/ElasticWaveEquation.cu:191-204):
//   1. source: txx, tyy, tzz at the source cell += dt*dt*s(it)
//      (OPT/ElasticWaveEquation.cu:206-221);
//   2. velocity update of every computed cell (OPT/ElasticWaveEquation.cu:234-526);
//   3. stress update of every computed cell (OPT/ElasticWaveEquation.cu:528-841);
//   4. receivers sample the fields (OPT/ElasticWaveEquation.cu:223-232; the
//      reference has one txx station, this oracle any list of components).
// Computed cells are [5, n-5) per axis; the 5-cell frame stays zero
// (OPT/ElasticMacro.h:30-39, 41).  Cells within `pml` of that range's faces
// are PML cells and use split fields, one split per derivative axis, the
// damped axes being those whose coordinate lies in a PML band
// (vertex/edge/surface regions OPT/ElasticWaveEquation.cu:47-108;
// split updates OPT/ElasticMacro.h:409-531).  The distance k used by the
// damping runs 1..pml from the inner edge of the band outwards
// (OPT/ElasticWaveEquation.cu:283-285, 297, 331).
//
// Floating-point contract.  The reference source leaves the rounding of
// `a += c*(x-y)` and similar statements to the compiler.  This oracle fixes
// one order and writes every fused multiply-add explicitly (std::fma); the
// CUDA kernels of the product use the same operations, so the FP32 oracle and
// the FP32 GPU path agree bit for bit on the same inputs.  Two deliberate
// departures from the literal reference expressions, both below one ulp of a
// damping coefficient: the damping profile uses r*r for powf(r, 2)
// (OPT/ElasticMacro.h:27), and each harmonic mu average takes 1/mu of each
// cell once (OPT/ElasticMacro.h:111-119 evaluates the same quotients).
// Build flags: -O3 -ffp-contract=off -fno-fast-math (see oracle/Makefile).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <xmmintrin.h>
#include <pmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/sgfd.h"

namespace {

constexpr int kHalo = 5;               // reference `order` (OPT/ElasticMacro.h:24)
constexpr float kTau = 4.3f;           // reference `tau`   (OPT/ElasticMacro.h:21)

enum { VX, VY, VZ, TXX, TYY, TZZ, TXY, TXZ, TYZ };
// Split-field ids: velocity (q, axis) then stress (OPT/ElasticMacro.h:335-363).
enum {
    S_VXX, S_VXY, S_VXZ, S_VYX, S_VYY, S_VYZ, S_VZX, S_VZY, S_VZZ,
    S_XXX, S_XXY, S_XXZ, S_YYX, S_YYY, S_YYZ, S_ZZX, S_ZZY, S_ZZZ,
    S_XYX, S_XYY, S_XZX, S_XZZ, S_YZY, S_YZZ, N_SPLIT
};

template <typename T> inline T fma_(T a, T b, T c) { return std::fma(a, b, c); }

// ---- 16-bit wavefield storage (sgfd_config.storage BF16 / F16) -------------
// The product stores each wavefield (and its PML splits) as 16-bit values h
// with a per-field power-of-two scale 2^e: stored = RN16(v * 2^-e), read back
// as float(h) * 2^e.  Arithmetic stays FP32.  These helpers restate that
// rounding on the CPU: round to nearest, ties to even, binary16 with
// subnormals and overflow to infinity, bfloat16 as the upper half of an
// FP32 word.

// v rounded to the nearest binary16 value, returned as float (IEEE: values
// from 65520 up overflow to infinity).
inline float rn_f16(float v) {
    if (!std::isfinite(v) || v == 0.0f) return v;
    const float av = std::fabs(v);
    if (av >= 65520.0f) return std::copysign(INFINITY, v);   // past the midpoint 65504 .. 2^16
    int e;
    std::frexp(av, &e);                       // av = m 2^e, m in [0.5, 1)
    const int ex = std::max(e - 1, -14);      // binade (subnormals share 2^-14's quantum)
    const float ulp = std::ldexp(1.0f, ex - 10);
    const float r = std::nearbyint(av / ulp) * ulp;   // av / ulp is exact; ties to even
    return std::copysign(r, v);
}
// v rounded to the nearest bfloat16 value (ties to even), returned as float.
inline float rn_bf16(float v) {
    if (!std::isfinite(v)) return v;
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}
// The storage rounding: binary16 saturates at +-65504 (a field outgrowing its
// scale between two rescales is clipped, not turned into infinity).
inline float store16(int storage, float w) {
    if (storage == SGFD_STORE_F16) return rn_f16(std::fmin(std::fmax(w, -65504.0f), 65504.0f));
    return rn_bf16(w);
}
// Steps after which the scales are re-chosen: it + 1 a power of two up to
// kRescaleEvery (the first steps of a run grow fast from zero), then every
// kRescaleEvery steps.  kScaleHead: the largest stored magnitude is put in
// [2^(kScaleHead-1), 2^kScaleHead), 256x below the binary16 maximum (room
// for growth until the next rescale) and 2^22 above its smallest normal.
constexpr int kRescaleEvery = 50;
constexpr int kScaleHead = 8;
inline bool rescale_step(int it) {
    const int n = it + 1;
    if (n <= 0) return false;
    return (n <= kRescaleEvery && (n & (n - 1)) == 0) || n % kRescaleEvery == 0;
}

struct Receiver { int x, y, z, comp; };

template <typename T>
struct Oracle {
    sgfd_config cfg{};
    int nx = 0, ny = 0, nz = 0;
    int64_t sy = 0, sz = 0, n = 0;
    std::vector<T> f[9];
    std::vector<T> b, lam, mu, rmu;   // rmu = 1/mu per cell
    std::vector<T> split[N_SPLIT];
    T c[5];
    T cs[3][5];      // FAST arithmetic: c_i / d_axis, rounded once
    bool fast = false;
    T dt, dx, dy, dz;
    int src_x = -1, src_y = -1, src_z = -1;
    std::vector<Receiver> rec;
    int nt = 0;
    std::vector<T> traces;
    bool ftz = false;
    // damping constants
    T q_refgpu[3];   // (0.5*dt*tau)   — multiplied by Vs, divided by d_axis, times poly
    T poly;          // 8/15 - 0.03 p + p^2/1500
    T q_logr;        // 0.5*dt*3*ln(1/R)/(2p)
    T q_refcpu[3];   // 0.5*dt*log10(1/R)*3.4*V/(p*d_axis)
    T qf[3];         // FAST: q constant pre-divided by the cell size
    // 16-bit storage emulation (FP32 oracle only): per-field scale exponents
    int storage = SGFD_STORE_F32;
    int scale_e[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    T pending_max[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // largest value written before rounding

    explicit Oracle(const sgfd_config &c_) : cfg(c_) {
        nx = cfg.nx; ny = cfg.ny; nz = cfg.nz;
        sy = nx; sz = (int64_t)nx * ny; n = sz * nz;
        for (auto &v : f) v.assign(n, T(0));
        b.assign(n, T(0)); lam.assign(n, T(0)); mu.assign(n, T(0)); rmu.assign(n, T(0));
        for (auto &v : split) v.assign(n, T(0));
        for (int i = 0; i < 5; ++i) c[i] = (T)cfg.coef[i];
        dt = (T)cfg.dt; dx = (T)cfg.dx; dy = (T)cfg.dy; dz = (T)cfg.dz;
        fast = cfg.arith == SGFD_ARITH_FAST;
        for (int i = 0; i < 5; ++i) { cs[0][i] = c[i] / dx; cs[1][i] = c[i] / dy; cs[2][i] = c[i] / dz; }
        const int p = cfg.pml;
        // (0.5f * delta.t) * tau  (OPT/ElasticMacro.h:26 in 1 - 0.5*dt*DAMPING)
        T h = (T)0.5f * dt * (T)kTau;
        q_refgpu[0] = q_refgpu[1] = q_refgpu[2] = h;
        // 8/15 - 0.03*pml + 1/1500*(pml*pml)   (OPT/ElasticMacro.h:26)
        poly = ((T)8.0f / (T)15.0f - (T)0.03f * (T)p) + ((T)1.0f / (T)1500.0f) * (T)(p * p);
        const double R = cfg.damping_R > 0 ? (double)cfg.damping_R : 1e-3;
        q_logr = (T)(0.5 * (double)cfg.dt * 3.0 * std::log(1.0 / R) / (2.0 * (double)p));
        const double dd[3] = {cfg.dx, cfg.dy, cfg.dz};
        for (int a = 0; a < 3; ++a)
            q_refcpu[a] = (T)(0.5 * (double)cfg.dt * std::log10(1.0 / R) * 3.4 *
                              (double)cfg.damping_vconst / ((double)p * dd[a]));
        const T d3[3] = {dx, dy, dz};
        for (int a = 0; a < 3; ++a)
            qf[a] = cfg.damping == SGFD_DAMP_LOGR ? q_logr / d3[a] : (h / d3[a]) * poly;
    }

    int64_t idx(int x, int y, int z) const { return x + (int64_t)y * sy + (int64_t)z * sz; }

    // Field each split belongs to (its scale group).
    static int split_field(int k) {
        static const int g[N_SPLIT] = {VX, VX, VX, VY, VY, VY, VZ, VZ, VZ, TXX, TXX, TXX, TYY, TYY, TYY,
                                       TZZ, TZZ, TZZ, TXY, TXY, TXZ, TXZ, TYZ, TYZ};
        return g[k];
    }
    // Stored value of v under field g's scale.
    T quant(T v, int g) const {
        const float sc = std::ldexp(1.0f, scale_e[g]), inv = std::ldexp(1.0f, -scale_e[g]);
        return (T)(store16(storage, (float)v * inv) * sc);
    }
    // Round fields [f0, f1] and their splits, just written by an update, to
    // the stored values.  On rescale steps first note each field's largest
    // written magnitude before rounding (a field whose values underflow the
    // current scale still gets a scale that fits them; the source injection
    // counts too, so that a run starting from zero fields gets going).
    void quantize_fields(int f0, int f1, bool track) {
        if (storage == SGFD_STORE_F32) return;
        if (track) {
            for (int g = f0; g <= f1; ++g) {
                T mx = 0;
                for (int64_t i = 0; i < n; ++i) mx = std::max(mx, (T)std::fabs(f[g][i]));
                for (int k = 0; k < N_SPLIT; ++k)
                    if (split_field(k) == g)
                        for (int64_t i = 0; i < n; ++i) mx = std::max(mx, (T)std::fabs(split[k][i]));
                pending_max[g] = std::max(pending_max[g], mx);
            }
        }
        for (int g = f0; g <= f1; ++g) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) f[g][i] = quant(f[g][i], g);
        }
        for (int k = 0; k < N_SPLIT; ++k) {
            const int g = split_field(k);
            if (g < f0 || g > f1) continue;
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) split[k][i] = quant(split[k][i], g);
        }
    }
    // Re-choose every field's scale so that the largest magnitude written in
    // this step lands in [2^(kScaleHead-1), 2^kScaleHead), then re-round the
    // stored values to the new scales.  Fields that wrote only zeros keep
    // their scale.
    void rescale() {
        for (int g = 0; g < 9; ++g) {
            const T mx = pending_max[g];
            pending_max[g] = 0;
            if (!(mx > 0) || !std::isfinite((float)mx)) continue;
            int e;
            std::frexp((float)mx, &e);            // mx in [2^(e-1), 2^e)
            scale_e[g] = std::min(100, std::max(-100, e - kScaleHead));
        }
        quantize_fields(0, 8, false);
    }

    // Forward staggered difference along `axis` (0,1,2 = x,y,z), stride s:
    // sum c_i (f[+1+i] - f[-i]) / d   (e.g. OPT/ElasticWaveEquation.cu:246, 250).
    // FAST arithmetic uses c_i/d and no division.
    inline T dfwd(const T *g, int64_t s, int axis) const {
        const T *k = fast ? cs[axis] : c;
        T d = 0;
        for (int i = 0; i < 5; ++i) d = fma_(k[i], g[(1 + i) * s] - g[-i * s], d);
        return fast ? d : d / (axis == 0 ? dx : axis == 1 ? dy : dz);
    }
    // Backward staggered difference: sum c_i (f[+i] - f[-1-i]) / d  (e.g. OPT/ElasticWaveEquation.cu:247)
    inline T dbwd(const T *g, int64_t s, int axis) const {
        const T *k = fast ? cs[axis] : c;
        T d = 0;
        for (int i = 0; i < 5; ++i) d = fma_(k[i], g[i * s] - g[(-1 - i) * s], d);
        return fast ? d : d / (axis == 0 ? dx : axis == 1 ? dy : dz);
    }
    // Harmonic average 4 / (r0 + r1 + r2 + r3) of four reciprocals; FAST takes
    // 4 * RN(1/s), which equals RN(4/s) exactly (a power-of-two scaling).
    inline T hmean(T r0, T r1, T r2, T r3) const {
        const T s = ((r0 + r1) + r2) + r3;
        return fast ? (T)4 * ((T)1 / s) : (T)4 / s;
    }

    // Damping band of coordinate i along an axis of length N: 0 if not in a
    // PML band, else k in 1..pml counted from the inner edge.
    inline int band(int i, int N) const {
        const int p = cfg.pml;
        if (i < kHalo + p) return (kHalo + p) - i;            // low side: end - i
        if (i >= N - kHalo - p) return i - (N - kHalo - p) + 1; // high side: i - start + 1
        return 0;
    }

    // (m, p) = (1 - q*r^2, 1 + q*r^2) for one damped axis; FAST returns
    // (m, RN(1/p)) and takes q from a constant pre-divided by the cell size.
    inline void damp(int axis, int k, int64_t ci, T &m, T &pp) const {
        const T d[3] = {dx, dy, dz};
        T q;
        if (cfg.damping == SGFD_DAMP_REFGPU) {
            // Vs = sqrt(mu*b) (OPT/ElasticWaveEquation.cu:282)
            T vs = std::sqrt(mu[ci] * b[ci]);
            q = fast ? vs * qf[axis] : ((q_refgpu[axis] * vs) / d[axis]) * poly;
        } else if (cfg.damping == SGFD_DAMP_LOGR) {
            T vp = std::sqrt(fma_((T)2, mu[ci], lam[ci]) * b[ci]);
            q = fast ? vp * qf[axis] : (q_logr * vp) / d[axis];
        } else {
            q = q_refcpu[axis];
        }
        T r = (T)k / (T)cfg.pml;
        T pw = r * r;
        m = fma_(-q, pw, (T)1);
        pp = fma_(q, pw, (T)1);
        if (fast) pp = (T)1 / pp;
    }

    void inject(T s, bool track) {
        if (src_x < 0) return;
        int64_t ci = idx(src_x, src_y, src_z);
        T v = (dt * dt) * s;   // deltaT * deltaT * sourceValue (OPT/ElasticWaveEquation.cu:213)
        f[TXX][ci] = f[TXX][ci] + v;
        f[TYY][ci] = f[TYY][ci] + v;
        f[TZZ][ci] = f[TZZ][ci] + v;
        if (storage != SGFD_STORE_F32)
            for (int g = TXX; g <= TZZ; ++g) {
                if (track) pending_max[g] = std::max(pending_max[g], (T)std::fabs(f[g][ci]));
                f[g][ci] = quant(f[g][ci], g);
            }
    }

    // One split update: damped -> (m*s + A*B)/p (FAST: times RN(1/p)); undamped -> s + A*B.
    inline T upd(T s, T A, T B, bool damped, T m, T p) const {
        if (!damped) return fma_(A, B, s);
        return fast ? fma_(m, s, A * B) * p : fma_(m, s, A * B) / p;
    }

    void velocity_cell(int x, int y, int z, int kx, int ky, int kz) {
        const int64_t ci = idx(x, y, z);
        const T *sxx = f[TXX].data() + ci, *syy = f[TYY].data() + ci, *szz = f[TZZ].data() + ci;
        const T *sxy = f[TXY].data() + ci, *sxz = f[TXZ].data() + ci, *syz = f[TYZ].data() + ci;
        const T *bb = b.data() + ci;
        // b averages (OPT/ElasticMacro.h:106-109)
        T bx = (bb[0] + bb[1]) / (T)2;
        T by = (bb[0] + bb[sy]) / (T)2;
        T bz = (bb[0] + bb[sz]) / (T)2;
        // derivatives (OPT/ElasticWaveEquation.cu:244-276)
        T xX = dfwd(sxx, 1, 0), xY = dbwd(sxy, sy, 1), xZ = dbwd(sxz, sz, 2);
        T yX = dbwd(sxy, 1, 0), yY = dfwd(syy, sy, 1), yZ = dbwd(syz, sz, 2);
        T zX = dbwd(sxz, 1, 0), zY = dbwd(syz, sy, 1), zZ = dfwd(szz, sz, 2);
        if (!(kx | ky | kz)) {
            // interior (OPT/ElasticWaveEquation.cu:253,265,277)
            f[VX][ci] = fma_(dt * bx, (xX + xY) + xZ, f[VX][ci]);
            f[VY][ci] = fma_(dt * by, (yX + yY) + yZ, f[VY][ci]);
            f[VZ][ci] = fma_(dt * bz, (zX + zY) + zZ, f[VZ][ci]);
            return;
        }
        T mx = 1, px = 1, my = 1, py = 1, mz = 1, pz = 1;
        if (kx) damp(0, kx, ci, mx, px);
        if (ky) damp(1, ky, ci, my, py);
        if (kz) damp(2, kz, ci, mz, pz);
        // PML split update (OPT/ElasticMacro.h:409-458).  REF quirk: x-average
        // buoyancy for all three components (OPT/ElasticMacro.h:424-456).
        const bool ref = cfg.quirks == SGFD_QUIRKS_REF;
        const T ax = dt * bx, ay = dt * (ref ? bx : by), az = dt * (ref ? bx : bz);
        T *s = nullptr;
        T a0, a1, a2;
        s = &split[S_VXX][ci]; a0 = *s = upd(*s, ax, xX, kx, mx, px);
        s = &split[S_VXY][ci]; a1 = *s = upd(*s, ax, xY, ky, my, py);
        s = &split[S_VXZ][ci]; a2 = *s = upd(*s, ax, xZ, kz, mz, pz);
        f[VX][ci] = (a0 + a1) + a2;
        s = &split[S_VYX][ci]; a0 = *s = upd(*s, ay, yX, kx, mx, px);
        s = &split[S_VYY][ci]; a1 = *s = upd(*s, ay, yY, ky, my, py);
        s = &split[S_VYZ][ci]; a2 = *s = upd(*s, ay, yZ, kz, mz, pz);
        f[VY][ci] = (a0 + a1) + a2;
        s = &split[S_VZX][ci]; a0 = *s = upd(*s, az, zX, kx, mx, px);
        s = &split[S_VZY][ci]; a1 = *s = upd(*s, az, zY, ky, my, py);
        s = &split[S_VZZ][ci]; a2 = *s = upd(*s, az, zZ, kz, mz, pz);
        f[VZ][ci] = (a0 + a1) + a2;
    }

    void stress_cell(int x, int y, int z, int kx, int ky, int kz) {
        const int64_t ci = idx(x, y, z);
        const T *vx = f[VX].data() + ci, *vy = f[VY].data() + ci, *vz = f[VZ].data() + ci;
        const T *r = rmu.data() + ci;
        // normal-stress derivatives (OPT/ElasticWaveEquation.cu:541-549)
        T dXx = dbwd(vx, 1, 0), dYy = dbwd(vy, sy, 1), dZz = dbwd(vz, sz, 2);
        // shear derivatives (OPT/ElasticWaveEquation.cu:565-591)
        T xyY = dfwd(vx, sy, 1), xyX = dfwd(vy, 1, 0);
        T xzZ = dfwd(vx, sz, 2), xzX = dfwd(vz, 1, 0);
        T yzZ = dfwd(vy, sz, 2), yzY = dfwd(vz, sy, 1);
        const T l = lam[ci];
        const T l2m = fma_((T)2, mu[ci], l);
        // harmonic mu averages (OPT/ElasticMacro.h:111-119); REF quirk in xz.
        const bool ref = cfg.quirks == SGFD_QUIRKS_REF;
        T mxy = hmean(r[0], r[1], r[sy], r[1 + sy]);
        T mxz = hmean(r[0], r[1], r[sz], ref ? r[1 + sy] : r[1 + sz]);
        T myz = hmean(r[0], r[sy], r[sz], r[sy + sz]);
        if (!(kx | ky | kz)) {
            // interior (OPT/ElasticWaveEquation.cu:550-592)
            f[TXX][ci] = fma_(dt, fma_(l2m, dXx, l * (dYy + dZz)), f[TXX][ci]);
            f[TYY][ci] = fma_(dt, fma_(l2m, dYy, l * (dXx + dZz)), f[TYY][ci]);
            f[TZZ][ci] = fma_(dt, fma_(l2m, dZz, l * (dXx + dYy)), f[TZZ][ci]);
            f[TXY][ci] = fma_(dt * mxy, xyY + xyX, f[TXY][ci]);
            f[TXZ][ci] = fma_(dt * mxz, xzZ + xzX, f[TXZ][ci]);
            f[TYZ][ci] = fma_(dt * myz, yzZ + yzY, f[TYZ][ci]);
            return;
        }
        T mx = 1, px = 1, my = 1, py = 1, mz = 1, pz = 1;
        if (kx) damp(0, kx, ci, mx, px);
        if (ky) damp(1, ky, ci, my, py);
        if (kz) damp(2, kz, ci, mz, pz);
        // PML split update (OPT/ElasticMacro.h:460-531)
        const T dl = dt * l2m;
        T *s; T a0, a1, a2;
        s = &split[S_XXX][ci]; a0 = *s = upd(*s, dl, dXx, kx, mx, px);
        s = &split[S_XXY][ci]; a1 = *s = upd(*s, dt, l * dYy, ky, my, py);
        s = &split[S_XXZ][ci]; a2 = *s = upd(*s, dt, l * dZz, kz, mz, pz);
        f[TXX][ci] = (a0 + a1) + a2;
        s = &split[S_YYX][ci]; a0 = *s = upd(*s, dt, l * dXx, kx, mx, px);
        s = &split[S_YYY][ci]; a1 = *s = upd(*s, dl, dYy, ky, my, py);
        s = &split[S_YYZ][ci]; a2 = *s = upd(*s, dt, l * dZz, kz, mz, pz);
        f[TYY][ci] = (a0 + a1) + a2;
        s = &split[S_ZZX][ci]; a0 = *s = upd(*s, dt, l * dXx, kx, mx, px);
        s = &split[S_ZZY][ci]; a1 = *s = upd(*s, dt, l * dYy, ky, my, py);
        s = &split[S_ZZZ][ci]; a2 = *s = upd(*s, dl, dZz, kz, mz, pz);
        f[TZZ][ci] = (a0 + a1) + a2;
        const T axy = dt * mxy, axz = dt * mxz, ayz = dt * myz;
        s = &split[S_XYX][ci]; a0 = *s = upd(*s, axy, xyX, kx, mx, px);
        s = &split[S_XYY][ci]; a1 = *s = upd(*s, axy, xyY, ky, my, py);
        f[TXY][ci] = a0 + a1;
        s = &split[S_XZX][ci]; a0 = *s = upd(*s, axz, xzX, kx, mx, px);
        s = &split[S_XZZ][ci]; a1 = *s = upd(*s, axz, xzZ, kz, mz, pz);
        f[TXZ][ci] = a0 + a1;
        s = &split[S_YZY][ci]; a0 = *s = upd(*s, ayz, yzY, ky, my, py);
        s = &split[S_YZZ][ci]; a1 = *s = upd(*s, ayz, yzZ, kz, mz, pz);
        f[TYZ][ci] = a0 + a1;
    }

    // Interior cells of one x-row, written as plain loops so the compiler
    // vectorises them; same per-cell operations as velocity_cell's interior
    // branch (OPT/ElasticWaveEquation.cu:241-278).
    void velocity_row(int y, int z, int x0, int x1) {
        const int64_t r0 = idx(0, y, z);
        const T *__restrict sxx = f[TXX].data() + r0, *__restrict syy = f[TYY].data() + r0;
        const T *__restrict szz = f[TZZ].data() + r0, *__restrict sxy = f[TXY].data() + r0;
        const T *__restrict sxz = f[TXZ].data() + r0, *__restrict syz = f[TYZ].data() + r0;
        const T *__restrict bb = b.data() + r0;
        T *__restrict vx = f[VX].data() + r0, *__restrict vy = f[VY].data() + r0, *__restrict vz = f[VZ].data() + r0;
        const int64_t Y = sy, Z = sz;
        const T *kx = fast ? cs[0] : c, *ky = fast ? cs[1] : c, *kz = fast ? cs[2] : c;
        const T qx = fast ? (T)1 : dx, qy = fast ? (T)1 : dy, qz = fast ? (T)1 : dz;
        for (int x = x0; x < x1; ++x) {
            T xX = 0, xY = 0, xZ = 0, yX = 0, yY = 0, yZ = 0, zX = 0, zY = 0, zZ = 0;
#pragma GCC unroll 5
            for (int i = 0; i < 5; ++i) {
                xX = fma_(kx[i], sxx[x + 1 + i] - sxx[x - i], xX);
                xY = fma_(ky[i], sxy[x + i * Y] - sxy[x - (1 + i) * Y], xY);
                xZ = fma_(kz[i], sxz[x + i * Z] - sxz[x - (1 + i) * Z], xZ);
                yX = fma_(kx[i], sxy[x + i] - sxy[x - 1 - i], yX);
                yY = fma_(ky[i], syy[x + (1 + i) * Y] - syy[x - i * Y], yY);
                yZ = fma_(kz[i], syz[x + i * Z] - syz[x - (1 + i) * Z], yZ);
                zX = fma_(kx[i], sxz[x + i] - sxz[x - 1 - i], zX);
                zY = fma_(ky[i], syz[x + i * Y] - syz[x - (1 + i) * Y], zY);
                zZ = fma_(kz[i], szz[x + (1 + i) * Z] - szz[x - i * Z], zZ);
            }
            // x / 1 is exact, so FAST takes the same code path
            xX /= qx; xY /= qy; xZ /= qz; yX /= qx; yY /= qy; yZ /= qz; zX /= qx; zY /= qy; zZ /= qz;
            const T bx = (bb[x] + bb[x + 1]) / (T)2, by = (bb[x] + bb[x + Y]) / (T)2, bz = (bb[x] + bb[x + Z]) / (T)2;
            vx[x] = fma_(dt * bx, (xX + xY) + xZ, vx[x]);
            vy[x] = fma_(dt * by, (yX + yY) + yZ, vy[x]);
            vz[x] = fma_(dt * bz, (zX + zY) + zZ, vz[x]);
        }
    }

    // Interior cells of one x-row for the stress update; same operations as
    // stress_cell's interior branch (OPT/ElasticWaveEquation.cu:535-593).
    void stress_row(int y, int z, int x0, int x1) {
        const int64_t r0 = idx(0, y, z);
        const T *__restrict vx = f[VX].data() + r0, *__restrict vy = f[VY].data() + r0, *__restrict vz = f[VZ].data() + r0;
        const T *__restrict la = lam.data() + r0, *__restrict m = mu.data() + r0, *__restrict r = rmu.data() + r0;
        T *__restrict sxx = f[TXX].data() + r0, *__restrict syy = f[TYY].data() + r0, *__restrict szz = f[TZZ].data() + r0;
        T *__restrict sxy = f[TXY].data() + r0, *__restrict sxz = f[TXZ].data() + r0, *__restrict syz = f[TYZ].data() + r0;
        const int64_t Y = sy, Z = sz;
        const int64_t q4 = cfg.quirks == SGFD_QUIRKS_REF ? 1 + Y : 1 + Z;
        const T *kx = fast ? cs[0] : c, *ky = fast ? cs[1] : c, *kz = fast ? cs[2] : c;
        const T qx = fast ? (T)1 : dx, qy = fast ? (T)1 : dy, qz = fast ? (T)1 : dz;
        for (int x = x0; x < x1; ++x) {
            T dXx = 0, dYy = 0, dZz = 0, xyY = 0, xyX = 0, xzZ = 0, xzX = 0, yzZ = 0, yzY = 0;
#pragma GCC unroll 5
            for (int i = 0; i < 5; ++i) {
                dXx = fma_(kx[i], vx[x + i] - vx[x - 1 - i], dXx);
                dYy = fma_(ky[i], vy[x + i * Y] - vy[x - (1 + i) * Y], dYy);
                dZz = fma_(kz[i], vz[x + i * Z] - vz[x - (1 + i) * Z], dZz);
                xyY = fma_(ky[i], vx[x + (1 + i) * Y] - vx[x - i * Y], xyY);
                xyX = fma_(kx[i], vy[x + 1 + i] - vy[x - i], xyX);
                xzZ = fma_(kz[i], vx[x + (1 + i) * Z] - vx[x - i * Z], xzZ);
                xzX = fma_(kx[i], vz[x + 1 + i] - vz[x - i], xzX);
                yzZ = fma_(kz[i], vy[x + (1 + i) * Z] - vy[x - i * Z], yzZ);
                yzY = fma_(ky[i], vz[x + (1 + i) * Y] - vz[x - i * Y], yzY);
            }
            dXx /= qx; dYy /= qy; dZz /= qz; xyY /= qy; xyX /= qx; xzZ /= qz; xzX /= qx; yzZ /= qz; yzY /= qy;
            const T l = la[x], l2m = fma_((T)2, m[x], l);
            sxx[x] = fma_(dt, fma_(l2m, dXx, l * (dYy + dZz)), sxx[x]);
            syy[x] = fma_(dt, fma_(l2m, dYy, l * (dXx + dZz)), syy[x]);
            szz[x] = fma_(dt, fma_(l2m, dZz, l * (dXx + dYy)), szz[x]);
            const T mxy = hmean(r[x], r[x + 1], r[x + Y], r[x + 1 + Y]);
            const T mxz = hmean(r[x], r[x + 1], r[x + Z], r[x + q4]);
            const T myz = hmean(r[x], r[x + Y], r[x + Z], r[x + Y + Z]);
            sxy[x] = fma_(dt * mxy, xyY + xyX, sxy[x]);
            sxz[x] = fma_(dt * mxz, xzZ + xzX, sxz[x]);
            syz[x] = fma_(dt * myz, yzZ + yzY, syz[x]);
        }
    }

    template <typename F, typename G>
    void sweep(F &&cell, G &&row) {
        const int z0 = kHalo, z1 = nz - kHalo;
#pragma omp parallel
        {
            if (ftz) _mm_setcsr(_mm_getcsr() | 0x8040);   // FTZ | DAZ
#pragma omp for schedule(dynamic, 1)
            for (int z = z0; z < z1; ++z) {
                const int kz = band(z, nz);
                for (int y = kHalo; y < ny - kHalo; ++y) {
                    const int ky = band(y, ny);
                    if (ky | kz) {
                        for (int x = kHalo; x < nx - kHalo; ++x) cell(x, y, z, band(x, nx), ky, kz);
                        continue;
                    }
                    const int xi0 = kHalo + cfg.pml, xi1 = nx - kHalo - cfg.pml;
                    for (int x = kHalo; x < xi0; ++x) cell(x, y, z, band(x, nx), 0, 0);
                    row(y, z, xi0, xi1);
                    for (int x = xi1; x < nx - kHalo; ++x) cell(x, y, z, band(x, nx), 0, 0);
                }
            }
            if (ftz) _mm_setcsr(_mm_getcsr() & ~0x8040u);
        }
    }

    void record(bool velocity_phase, int it) {
        if (it < 0 || it >= nt) return;
        for (size_t r = 0; r < rec.size(); ++r) {
            const Receiver &q = rec[r];
            const bool is_v = q.comp <= VZ;
            if (is_v != velocity_phase) continue;
            traces[r * (size_t)nt + it] = f[q.comp][idx(q.x, q.y, q.z)];
        }
    }

    void step(int it, T s) {
        const bool rs = storage != SGFD_STORE_F32 && rescale_step(it);
        inject(s, rs);
        sweep([this](int x, int y, int z, int kx, int ky, int kz) { velocity_cell(x, y, z, kx, ky, kz); },
              [this](int y, int z, int x0, int x1) { velocity_row(y, z, x0, x1); });
        quantize_fields(VX, VZ, rs);
        record(true, it);
        sweep([this](int x, int y, int z, int kx, int ky, int kz) { stress_cell(x, y, z, kx, ky, kz); },
              [this](int y, int z, int x0, int x1) { stress_row(y, z, x0, x1); });
        quantize_fields(TXX, TYZ, rs);
        record(false, it);
        if (rs) rescale();
    }
};

struct Handle {
    int fp64 = 0;
    std::unique_ptr<Oracle<float>> f32;
    std::unique_ptr<Oracle<double>> f64;
    std::string err;
};

template <typename Fn>
int dispatch(Handle *h, Fn &&fn) {
    if (!h) return SGFD_ERR_INVALID;
    if (h->fp64) return fn(*h->f64);
    return fn(*h->f32);
}

}  // namespace

extern "C" {

void *sgo_create(const sgfd_config *cfg, int fp64) {
    if (!cfg || cfg->nx < 11 || cfg->ny < 11 || cfg->nz < 11 || cfg->pml < 0) return nullptr;
    if (2 * (cfg->pml + kHalo) > std::min({cfg->nx, cfg->ny, cfg->nz})) return nullptr;
    auto *h = new Handle();
    h->fp64 = fp64;
    if (fp64) h->f64.reset(new Oracle<double>(*cfg));
    else {
        h->f32.reset(new Oracle<float>(*cfg));
        h->f32->storage = cfg->storage;   // 16-bit storage emulated in FP32 runs only
    }
    return h;
}

void sgo_destroy(void *p) { delete static_cast<Handle *>(p); }

int sgo_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int sgo_set_ftz(void *p, int on) {
    return dispatch(static_cast<Handle *>(p), [&](auto &o) { o.ftz = on != 0; return 0; });
}

int sgo_set_medium(void *p, const float *bu, const float *la, const float *mu) {
    return dispatch(static_cast<Handle *>(p), [&](auto &o) {
        using T = typename std::remove_reference<decltype(o.b[0])>::type;
        for (int64_t i = 0; i < o.n; ++i) {
            o.b[i] = (T)bu[i]; o.lam[i] = (T)la[i]; o.mu[i] = (T)mu[i];
            o.rmu[i] = (T)1 / o.mu[i];   // 1 / mu  (OPT/ElasticMacro.h:112)
        }
        return 0;
    });
}

int sgo_set_source(void *p, int x, int y, int z) {
    return dispatch(static_cast<Handle *>(p), [&](auto &o) {
        if (x < kHalo || y < kHalo || z < kHalo || x >= o.nx - kHalo || y >= o.ny - kHalo || z >= o.nz - kHalo)
            return (int)SGFD_ERR_INVALID;
        o.src_x = x; o.src_y = y; o.src_z = z;
        return 0;
    });
}

int sgo_set_receivers(void *p, int nrec, const int *xyz, const int *comp, int nt) {
    return dispatch(static_cast<Handle *>(p), [&](auto &o) {
        o.rec.clear();
        for (int r = 0; r < nrec; ++r) {
            Receiver q{xyz[3 * r], xyz[3 * r + 1], xyz[3 * r + 2], comp[r]};
            if (q.x < 0 || q.y < 0 || q.z < 0 || q.x >= o.nx || q.y >= o.ny || q.z >= o.nz || q.comp < 0 || q.comp > 8)
                return (int)SGFD_ERR_INVALID;
            o.rec.push_back(q);
        }
        o.nt = nt;
        o.traces.assign((size_t)nrec * nt, 0);
        return 0;
    });
}

// Steps it0..it0+nsteps-1 with source values wavelet[it] (wavelet indexed by it).
int sgo_run(void *p, int it0, int nsteps, const double *wavelet) {
    return dispatch(static_cast<Handle *>(p), [&](auto &o) {
        using T = typename std::remove_reference<decltype(o.b[0])>::type;
        for (int it = it0; it < it0 + nsteps; ++it) o.step(it, (T)wavelet[it]);
        return 0;
    });
}

int sgo_get_traces(void *p, double *out) {
    return dispatch(static_cast<Handle *>(p), [&](auto &o) {
        for (size_t i = 0; i < o.traces.size(); ++i) out[i] = (double)o.traces[i];
        return 0;
    });
}

int sgo_get_field(void *p, int field, double *out) {
    return dispatch(static_cast<Handle *>(p), [&](auto &o) {
        if (field < 0 || field > 8) return (int)SGFD_ERR_INVALID;
        for (int64_t i = 0; i < o.n; ++i) out[i] = (double)o.f[field][i];
        return 0;
    });
}

// Overwrite one wavefield from n float values (GRID, x fastest): initial
// conditions, as sgfd_set_field does on the GPU.
int sgo_set_field(void *p, int field, const float *in) {
    return dispatch(static_cast<Handle *>(p), [&](auto &o) {
        if (field < 0 || field > 8) return (int)SGFD_ERR_INVALID;
        for (int64_t i = 0; i < o.n; ++i) o.f[field][i] = in[i];
        return 0;
    });
}

// The 16-bit roundings of the storage emulation, for checking against numpy.
void sgo_round16(int storage, const float *in, float *out, int64_t n) {
    for (int64_t i = 0; i < n; ++i) out[i] = storage == SGFD_STORE_F16 ? rn_f16(in[i]) : rn_bf16(in[i]);
}

// Scale exponents of the 9 fields (16-bit storage emulation).
int sgo_scale_exponents(void *p, int *out) {
    auto *h = static_cast<Handle *>(p);
    if (!h || h->fp64) return SGFD_ERR_INVALID;
    for (int g = 0; g < 9; ++g) out[g] = h->f32->scale_e[g];
    return 0;
}

// Reference Ricker wavelet (OPT/ElasticWaveEquation.cu:184-189), evaluated in
// float exactly as the reference host code does: pow(float, 2) promotes to
// double, whose product of two floats is exact, then rounds to float.
float sgo_ricker_ref(float f0, float dt, int it) {
    const float pi = 3.1415926f;                       // OPT/ElasticMacro.h:19
    float t0 = std::ceil(1.0f / (f0 * dt));
    float a = pi * f0 * (((float)it - t0) * dt - 1.0f / f0);
    float tmp = (float)((double)a * (double)a);
    return (1.0f - 2.0f * tmp) * std::exp(-tmp);
}

}  // extern "C"
