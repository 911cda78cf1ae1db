// ug_frames.cu -- past-light-cone frame baking of a packed universe (2+1).
//
// For each instant z_obs and observer, the pulse centre is frozen at the
// observer's comoving position and the universe is rewound while a front
// expands (cuda/frame_bake.cu:1-40): front "speed" (conformal, speed c),
// "fit" (c = -1/eta(z_min)) or "budget" (wiggle-budget reach).  Every torus
// image (2nx, 2ny), |n| <= K, of every worldline is walked along the rewind
// grid for sign changes of dist(pos + shift - centre) - chi_front and each
// crossing is refined by 24 bisection steps with fresh evaluations
// (frame_bake.cu:281-371).  Hits are (src, dx, dy, chi, z_emit); optionally
// they are histogrammed into a bins x bins uint32 density grid per frame over
// [-chi_max, chi_max]^2 (no reference counterpart; the reference draws
// scatter plots, plots/render_frames.py:47-110).
//
// Evaluation: X(z) = [a2 sin z + sum_j a_j (sin(b_j z + f_j) - sin f_j)] / sin z
// (frame_bake.cu:201-212).  Full-band dumps evaluate sum_j a_j sin(b_j z + f_j)
// as Im P(e^{iz}) with P(w) = sum_b (a_b e^{i f_b}) w^b by complex Horner --
// one sincos per evaluation instead of one per term; few-term dumps sum the
// terms directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "ug_frames.cuh"

namespace ug {

int set_error(int code, const char* msg);

namespace {

constexpr int kGridRows = 420;     // rewind grid (frame_bake.cu:71)
constexpr int kBisect = 24;        // bisection steps (frame_bake.cu:72)
constexpr int kBudgetCap = 4000;   // budget rewind-grid cap (frame_bake.cu:73)
constexpr double kPiF = 3.14159265358979323846;

struct FPaths {
    int n, nw, bmax;
    int horner;            // 1: complex Horner over b = 0..bmax; 0: per-term sums
    const double* a2;      // [n][2]
    const double* s0;      // [n][2]  sum_j a_j sin f_j
    const double* a;       // [n][2][nw]
    const double* b;       // [n][2][nw]
    const double* f;       // [n][2][nw]
    const double2* coef;   // [n][2][bmax+1] a_b e^{i f_b} (Horner form)
};

struct FFront {
    int budget, cheb, M, bMax;
    double spd, zObs, etaObs, chiMax;
};

__host__ __device__ inline double wiggle_direct(const double* a, const double* b, const double* f, int nw,
                                                double z) {
    double s = 0.0;
    for (int j = 0; j < nw; j++) s += a[j] * sin(b[j] * z + f[j]);
    return s;
}

__device__ inline double wiggle_horner(const double2* c, int bmax, double z) {
    double sz, cz;
    sincos(z, &sz, &cz);
    double pr = c[bmax].x, pi = c[bmax].y;
    for (int k = bmax - 1; k >= 0; k--) {
        const double nr = fma(pr, cz, fma(-pi, sz, c[k].x));
        const double ni = fma(pr, sz, fma(pi, cz, c[k].y));
        pr = nr;
        pi = ni;
    }
    return pi;
}

__device__ inline void comov(const FPaths& P, int p, double z, double* X, double* Y) {
    const double s = sin(z);
    double w[2];
    for (int ax = 0; ax < 2; ax++) {
        const size_t o = ((size_t)p * 2 + ax);
        w[ax] = P.horner ? wiggle_horner(P.coef + o * (P.bmax + 1), P.bmax, z)
                         : wiggle_direct(P.a + o * P.nw, P.b + o * P.nw, P.f + o * P.nw, P.nw, z);
    }
    *X = (P.a2[(size_t)p * 2] * s + w[0] - P.s0[(size_t)p * 2]) / s;
    *Y = (P.a2[(size_t)p * 2 + 1] * s + w[1] - P.s0[(size_t)p * 2 + 1]) / s;
}

// Wiggle-budget reach of the front (frame_bake.cu:236-251).
__host__ __device__ inline double reach_of(double z, double zObs, int bMax) {
    const double s = sin(z), sObs = sin(zObs);
    double best = 0.0;
    for (int b = 2; b <= bMax; b++) {
        const double da = (cos(b * z) - 1.0) / (b * s) - (cos(b * zObs) - 1.0) / (b * sObs);
        const double db = sin(b * z) / (b * s) - sin(b * zObs) / (b * sObs);
        const double d = (b % 2 == 0) ? sqrt(da * da + db * db) : fabs(db);
        best = d > best ? d : best;
    }
    return best;
}

__device__ inline double metric(double dx, double dy, int cheb) {
    return cheb ? fmax(fabs(dx), fabs(dy)) : sqrt(dx * dx + dy * dy);
}

// Rewind-grid positions, one thread per (path, 4 consecutive rows): four
// independent Horner chains per thread (each row the same operations as comov).
__global__ void k_fb_grid(FPaths P, int M, const double* zg, double* px, double* py) {
    const int R = M + 1, G = (R + 3) / 4;
    const int64_t total = (int64_t)P.n * G;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(i / G), r0 = (int)(i % G) * 4;
        double z[4], s[4], w[2][4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            z[q] = zg[min(r0 + q, R - 1)];
            s[q] = sin(z[q]);
        }
        for (int ax = 0; ax < 2; ax++) {
            const size_t o = (size_t)p * 2 + ax;
            if (P.horner) {
                const double2* c = P.coef + o * (P.bmax + 1);
                double sz[4], cz[4], pr[4], pi[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    sincos(z[q], &sz[q], &cz[q]);
                    pr[q] = c[P.bmax].x;
                    pi[q] = c[P.bmax].y;
                }
                for (int k = P.bmax - 1; k >= 0; k--) {
                    const double2 ck = c[k];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const double nr = fma(pr[q], cz[q], fma(-pi[q], sz[q], ck.x));
                        const double ni = fma(pr[q], sz[q], fma(pi[q], cz[q], ck.y));
                        pr[q] = nr;
                        pi[q] = ni;
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; q++) w[ax][q] = pi[q];
            } else {
#pragma unroll
                for (int q = 0; q < 4; q++)
                    w[ax][q] = wiggle_direct(P.a + o * P.nw, P.b + o * P.nw, P.f + o * P.nw, P.nw, z[q]);
            }
        }
        const double a2x = P.a2[(size_t)p * 2], a2y = P.a2[(size_t)p * 2 + 1];
        const double s0x = P.s0[(size_t)p * 2], s0y = P.s0[(size_t)p * 2 + 1];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (r0 + q >= R) break;
            const int64_t at = (int64_t)p * R + r0 + q;
            px[at] = (a2x * s[q] + w[0][q] - s0x) / s[q];
            py[at] = (a2y * s[q] + w[1][q] - s0y) / s[q];
        }
    }
}

// A sign change of dist(image) - chi_front between rewind rows i-1 and i.
struct FCross {
    int32_t p;
    int16_t nx, ny;
    int32_t i;
    int32_t inside;  // the image was inside the front at row i-1
};

// One thread per (path, torus image): walks the rewind grid and records every
// crossing; the bisections run in k_fb_refine, one thread per crossing, so no
// warp waits for a single lane's refinement.
__global__ void k_fb_cross(FPaths P, FFront F, double ox, double oy, int K, int obsIdx, const double* chig,
                           const double* px, const double* py, FCross* cross, unsigned long long* count,
                           unsigned long long cap) {
    const int side = 2 * K + 1;
    const int64_t total = (int64_t)P.n * side * side;
    for (int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; tid < total;
         tid += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(tid / (side * side));
        const int sh = (int)(tid % (side * side));
        const int nx = sh % side - K, ny = sh / side - K;
        const double bx = 2.0 * nx - ox, by = 2.0 * ny - oy;
        // rows the front cannot reach for this image (comoving coords stay within +-2)
        const double dmin = fmax(0.0, 2.0 * fmax(fabs((double)nx), fabs((double)ny)) - 4.0);
        if (dmin >= F.chiMax) continue;
        const int i0 = F.budget ? 1 : max(1, (int)ceil(dmin * F.M / F.chiMax));
        if (i0 > F.M) continue;
        const int64_t row = (int64_t)p * (F.M + 1);
        double prev = metric(px[row + i0 - 1] + bx, py[row + i0 - 1] + by, F.cheb) - chig[i0 - 1];
        // the observer sits on the front at chi = 0: keep its own image inside
        if (p == obsIdx && nx == 0 && ny == 0 && i0 == 1 && fabs(prev) < 1e-9)
            prev = -1e-12;
        else if (prev == 0.0)
            prev = 1e-12;
        for (int i = i0; i <= F.M; i++) {
            const double g = metric(px[row + i] + bx, py[row + i] + by, F.cheb) - chig[i];
            if ((prev < 0.0) != (g < 0.0)) {
                const unsigned long long slot = atomicAdd(count, 1ull);
                if (slot < cap) cross[slot] = FCross{p, (int16_t)nx, (int16_t)ny, i, prev < 0.0 ? 1 : 0};
            }
            prev = g;
        }
    }
}

// One thread per crossing: 24 bisection steps with fresh evaluations
// (frame_bake.cu:281-371), hit slot = crossing slot.
__global__ void k_fb_refine(FPaths P, FFront F, double ox, double oy, const double* zg, const double* chig,
                            const FCross* cross, const unsigned long long* count, unsigned long long cap,
                            ug_hit* hits) {
    const unsigned long long c = *count;
    const int64_t n = (int64_t)(c < cap ? c : cap);
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const FCross x = cross[k];
        const int p = x.p, i = x.i;
        const bool inside = x.inside != 0;
        const double bx = 2.0 * x.nx - ox, by = 2.0 * x.ny - oy;
        double chi, zEmit, qx, qy;
        if (F.budget) {
            double lo = zg[i - 1], hi = zg[i];
            for (int it = 0; it < kBisect; it++) {
                const double mid = (lo + hi) / 2.0;
                comov(P, p, mid, &qx, &qy);
                const double gm = metric(qx + bx, qy + by, F.cheb) - reach_of(mid, F.zObs, F.bMax);
                if ((gm < 0.0) == inside)
                    lo = mid;
                else
                    hi = mid;
            }
            zEmit = (lo + hi) / 2.0;
            chi = reach_of(zEmit, F.zObs, F.bMax);
        } else {
            double lo = chig[i - 1], hi = chig[i];
            for (int it = 0; it < kBisect; it++) {
                const double mid = (lo + hi) / 2.0;
                comov(P, p, 2.0 * atan(exp(F.etaObs - mid / F.spd)), &qx, &qy);
                const double gm = metric(qx + bx, qy + by, F.cheb) - mid;
                if ((gm < 0.0) == inside)
                    lo = mid;
                else
                    hi = mid;
            }
            chi = (lo + hi) / 2.0;
            zEmit = 2.0 * atan(exp(F.etaObs - chi / F.spd));
        }
        comov(P, p, zEmit, &qx, &qy);
        ug_hit h;
        h.src = (uint32_t)p;
        h.dx = (float)(qx + bx);
        h.dy = (float)(qy + by);
        h.chi = (float)chi;
        h.z_emit = (float)zEmit;
        hits[k] = h;
    }
}

// Density scatter: hit offsets binned over the closed square [-chi_max, chi_max]^2.
// Every hit lies on a front of radius chi <= chi_max, so every hit is counted:
// an offset that FP32 rounding puts a hair past an edge goes to the edge bin.
// Privatised by bands of rows: CTA b owns rows [b rows, (b+1) rows) of the grid in
// shared memory, streams all hits of the frame (coalesced, L2-resident), counts
// the ones in its band with shared-memory atomics and writes its band once,
// coalesced -- no global atomics and no separate clear of the grid.  The hit count
// is n, or *count (capped at cap) when count is given (read on the device).
__global__ void k_fb_density(const ug_hit* __restrict__ hits, int64_t n, const unsigned long long* count,
                             unsigned long long cap, double chiMax, int bins, int rows, uint32_t* grid) {
    extern __shared__ uint32_t band[];
    const int r0 = blockIdx.x * rows;
    const int nr = min(rows, bins - r0);
    const int cells = nr * bins;
    for (int i = threadIdx.x; i < cells; i += blockDim.x) band[i] = 0u;
    __syncthreads();
    if (count) {
        const unsigned long long c = *count;
        n = (int64_t)(c < cap ? c : cap);
    }
    const float inv = (float)(bins / (2.0 * chiMax));
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const ug_hit h = hits[i];
        int cy = (int)floorf((h.dy + (float)chiMax) * inv);
        cy = cy < 0 ? 0 : (cy >= bins ? bins - 1 : cy);
        if (cy < r0 || cy >= r0 + nr) continue;
        int cx = (int)floorf((h.dx + (float)chiMax) * inv);
        cx = cx < 0 ? 0 : (cx >= bins ? bins - 1 : cx);
        atomicAdd(&band[(cy - r0) * bins + cx], 1u);
    }
    __syncthreads();
    uint32_t* out = grid + (size_t)r0 * bins;
    for (int i = threadIdx.x; i < cells; i += blockDim.x) out[i] = band[i];
}

// Rows per density band: bands of at most 48 KB of shared memory.
inline int density_rows(int bins) { return std::max(1, std::min(bins, 12288 / bins)); }

inline void launch_density(const ug_hit* hits, int64_t n, const unsigned long long* count,
                           unsigned long long cap, double chiMax, int bins, uint32_t* grid, cudaStream_t st) {
    const int rows = density_rows(bins);
    const int bands = (bins + rows - 1) / rows;
    k_fb_density<<<bands, 512, (size_t)rows * bins * 4, st>>>(hits, n, count, cap, chiMax, bins, rows, grid);
}

double h_eta(double z) { return log(tan(z / 2.0)); }

// Host comoving position and velocity of a path (frame_bake.cu:201-228).
void h_comov(const std::vector<double>& a2, const std::vector<double>& a, const std::vector<double>& b,
             const std::vector<double>& f, int nw, int p, double z, double* X, double* Y, double* VX,
             double* VY) {
    const double s = sin(z), c = cos(z);
    double xx[2], dd[2];
    for (int ax = 0; ax < 2; ax++) {
        xx[ax] = a2[(size_t)p * 2 + ax] * s;
        dd[ax] = a2[(size_t)p * 2 + ax] * c;
        for (int j = 0; j < nw; j++) {
            const size_t o = ((size_t)p * 2 + ax) * nw + j;
            xx[ax] += a[o] * (sin(b[o] * z + f[o]) - sin(f[o]));
            dd[ax] += a[o] * b[o] * cos(b[o] * z + f[o]);
        }
    }
    *X = xx[0] / s;
    *Y = xx[1] / s;
    *VX = (dd[0] * s - xx[0] * c) / (s * s);
    *VY = (dd[1] * s - xx[1] * c) / (s * s);
}

struct DevBuf {
    std::vector<void*> p;
    ~DevBuf() {
        for (void* q : p) cudaFree(q);
    }
    template <class T>
    T* get(size_t n) {
        void* q = nullptr;
        if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
        p.push_back(q);
        return (T*)q;
    }
};

// Per (path, axis): s0 = sum_j a_j sin f_j and the Horner coefficients
// a_b e^{i f_b} (coef zeroed by the caller; frequencies are unique per axis).
__global__ void k_fb_prep(int n, int nw, int bmax, int horner, const double* a, const double* b,
                          const double* f, double* s0, double2* coef) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)n * 2;
         i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < nw; j++) {
            const int64_t o = i * nw + j;
            const double sf = sin(f[o]);
            acc += a[o] * sf;
            if (horner) {
                double2& c = coef[i * (bmax + 1) + (int)b[o]];
                c.x += a[o] * cos(f[o]);
                c.y += a[o] * sf;
            }
        }
        s0[i] = acc;
    }
}

// Dump-layout parameters from the packer (2+1): b as double for the direct sums.
__global__ void k_fb_from_params(int64_t m, const int32_t* bi, double* bd) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        bd[i] = (double)bi[i];
}

// One observer path's parameters on the host (for its comoving position and velocity).
struct ObsPath {
    std::vector<double> a2, a, b, f;  // [2], [2][nw] x3
};

int check_cfg(const ug_frames_cfg* cfg, ug_frames_out* out, int n) {
    if (!cfg || !out || n < 1) return set_error(UG_EINVAL, "frame_bake: bad arguments");
    if (cfg->front < 0 || cfg->front > 2) return set_error(UG_EINVAL, "--front must be speed|fit|budget");
    if (cfg->n_frames < 1 || cfg->n_obs < 1) return set_error(UG_EINVAL, "need >= 1 frame and observer");
    for (int o = 0; o < cfg->n_obs; o++)
        if (cfg->obs_type[o] == 0 && (cfg->obs_path[o] < 0 || cfg->obs_path[o] >= n))
            return set_error(UG_EINVAL, "observer path out of range");
    return UG_OK;
}

// The frame loop over device-resident paths (dump layout, b as double).  With a hit
// buffer the hits of every (frame, observer) come back sorted by (chi, src); without
// one only counts and densities do, and no step waits for the host.
int bake_device(const ug_frames_cfg* cfg, int n, int nw, int bMax, const double* dA2, const double* dA,
                const double* dB, const double* dF, const std::vector<ObsPath>& obs, ug_frames_out* out,
                cudaStream_t st) {
    DevBuf buf;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // Horner when the band is dense enough that one polynomial beats nw sines
    const int horner = (bMax <= 4 * nw) ? 1 : 0;
    double* dS0 = buf.get<double>((size_t)n * 2);
    double2* dC = buf.get<double2>(horner ? (size_t)n * 2 * (bMax + 1) : 1);
    const int Mmax = std::min(kBudgetCap, std::max(kGridRows, 2 * bMax));
    const int NF = cfg->n_frames, NO = cfg->n_obs;
    double* dZg = buf.get<double>((size_t)NF * (Mmax + 1));
    double* dChig = buf.get<double>((size_t)NF * (Mmax + 1));
    double* dPx = buf.get<double>((size_t)n * (Mmax + 1));
    double* dPy = buf.get<double>((size_t)n * (Mmax + 1));
    const bool want_hits = out->hits != nullptr;
    const bool want_density = cfg->density_bins > 0 && out->density;
    const size_t bins2 = want_density ? (size_t)cfg->density_bins * cfg->density_bins : 0;
    // densities: per (frame, observer) when hits come back one launch at a time,
    // all of them on the device otherwise (one copy at the end)
    uint32_t* dDen = want_density ? buf.get<uint32_t>(want_hits ? bins2 : bins2 * NF * NO) : nullptr;
    const unsigned long long hitCap = 1ull << 24;  // per (frame, observer) launch, frame_bake.cu:515
    ug_hit* dHits = buf.get<ug_hit>(hitCap);
    FCross* dCross = buf.get<FCross>(hitCap);
    unsigned long long* dCount = buf.get<unsigned long long>((size_t)NF * NO);
    if (!dS0 || !dC || !dZg || !dChig || !dPx || !dPy || !dHits || !dCross || !dCount || (want_density && !dDen))
        return set_error(UG_ENOMEM, "frame_bake: device allocation failed");
    if (horner) cudaMemsetAsync(dC, 0, (size_t)n * 2 * (bMax + 1) * sizeof(double2), st);
    k_fb_prep<<<(int)std::min<int64_t>(((int64_t)n * 2 + 127) / 128, 65536), 128, 0, st>>>(n, nw, bMax, horner, dA,
                                                                                           dB, dF, dS0, dC);
    cudaMemsetAsync(dCount, 0, (size_t)NF * NO * sizeof(unsigned long long), st);
    FPaths P{n, nw, bMax, horner, dA2, dS0, dA, dB, dF, dC};
    const double zMin = std::max(2e-3, cfg->zmin_pi * kPiF);
    // fronts and rewind grids of every frame, uploaded once
    std::vector<FFront> fronts(NF);
    std::vector<int> Ks(NF);
    std::vector<double> zgAll((size_t)NF * (Mmax + 1)), chigAll((size_t)NF * (Mmax + 1));
    for (int fi = 0; fi < NF; fi++) {
        const double frac = NF == 1 ? 0.0 : (double)fi / (NF - 1);
        const double zObs = std::min((cfg->from_pi + (cfg->to_pi - cfg->from_pi) * frac) * kPiF, kPiF - 1e-3);
        if (zMin >= zObs) return set_error(UG_EINVAL, "rewind floor >= z_obs");
        FFront& F = fronts[fi];
        F = FFront{};
        F.budget = cfg->front == 2;
        F.cheb = F.budget || cfg->cheb;
        F.zObs = zObs;
        F.etaObs = h_eta(zObs);
        F.spd = cfg->front == 0 ? std::max(1e-3, cfg->speed) : -1.0 / h_eta(zMin);
        F.bMax = bMax;
        F.M = F.budget ? std::min(kBudgetCap, std::max(kGridRows, 2 * bMax)) : kGridRows;
        double* zg = zgAll.data() + (size_t)fi * (Mmax + 1);
        double* chig = chigAll.data() + (size_t)fi * (Mmax + 1);
        if (F.budget) {
            F.chiMax = 0.0;
            for (int i = 0; i <= F.M; i++) {
                zg[i] = zObs - (zObs - zMin) * i / F.M;
                chig[i] = reach_of(zg[i], zObs, bMax);
                F.chiMax = std::max(F.chiMax, chig[i]);
            }
        } else {
            F.chiMax = F.spd * (F.etaObs - h_eta(zMin));
            for (int i = 0; i <= F.M; i++) {
                chig[i] = F.chiMax * i / F.M;
                zg[i] = 2.0 * atan(exp(F.etaObs - chig[i] / F.spd));
            }
        }
        Ks[fi] = cfg->wraps >= 0 ? cfg->wraps : (int)ceil((F.chiMax + 4.0) / 2.0);
        if (out->frame_meta) {
            out->frame_meta[fi * 3 + 0] = zObs;
            out->frame_meta[fi * 3 + 1] = F.chiMax;
            out->frame_meta[fi * 3 + 2] = Ks[fi];
        }
    }
    cudaMemcpyAsync(dZg, zgAll.data(), zgAll.size() * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dChig, chigAll.data(), chigAll.size() * 8, cudaMemcpyHostToDevice, st);
    int64_t written = 0;
    out->hits_total = 0;
    std::vector<ug_hit> hh;
    for (int fi = 0; fi < NF; fi++) {
        const FFront& F = fronts[fi];
        const int K = Ks[fi];
        const double* zg = dZg + (size_t)fi * (Mmax + 1);
        const double* chig = dChig + (size_t)fi * (Mmax + 1);
        {
            const int64_t tot = (int64_t)n * ((F.M + 1 + 3) / 4);
            k_fb_grid<<<(int)std::min<int64_t>((tot + 127) / 128, 65536), 128, 0, st>>>(P, F.M, zg, dPx, dPy);
        }
        for (int o = 0; o < NO; o++) {
            double ox, oy, bxv = 0.0, byv = 0.0;
            if (cfg->obs_type[o] == 0) {
                double vx, vy;
                const ObsPath& q = obs[o];
                h_comov(q.a2, q.a, q.b, q.f, nw, 0, F.zObs, &ox, &oy, &vx, &vy);
                bxv = sin(F.zObs) * vx / F.spd;
                byv = sin(F.zObs) * vy / F.spd;
            } else {
                ox = cfg->obs_xy[2 * o];
                oy = cfg->obs_xy[2 * o + 1];
            }
            if (out->obs_meta) {
                double* m = out->obs_meta + ((size_t)fi * NO + o) * 4;
                m[0] = ox;
                m[1] = oy;
                m[2] = bxv;
                m[3] = byv;
            }
            unsigned long long* cnt = dCount + (size_t)fi * NO + o;
            const int side = 2 * K + 1;
            const int64_t tot = (int64_t)n * side * side;
            k_fb_cross<<<(int)std::min<int64_t>((tot + 127) / 128, 1 << 20), 128, 0, st>>>(
                P, F, ox, oy, K, cfg->obs_type[o] == 0 ? cfg->obs_path[o] : -1, chig, dPx, dPy, dCross, cnt, hitCap);
            k_fb_refine<<<nsm * 8, 128, 0, st>>>(P, F, ox, oy, zg, chig, dCross, cnt, hitCap, dHits);
            if (!want_hits) {
                if (want_density)
                    launch_density(dHits, 0, cnt, hitCap, F.chiMax, cfg->density_bins,
                                   dDen + ((size_t)fi * NO + o) * bins2, st);
                continue;
            }
            unsigned long long nh = 0;
            cudaError_t e = cudaMemcpyAsync(&nh, cnt, 8, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                std::string m = std::string("frame_bake: ") + cudaGetErrorString(e);
                return set_error(UG_ECUDA, m.c_str());
            }
            if (nh > hitCap) return set_error(UG_ECAP, "frame_bake: hit cap overflow (lower the wraps)");
            if (want_density) {
                launch_density(dHits, (int64_t)nh, nullptr, hitCap, F.chiMax, cfg->density_bins, dDen, st);
                cudaMemcpyAsync(out->density + ((size_t)fi * NO + o) * bins2, dDen, bins2 * 4, cudaMemcpyDeviceToHost,
                                st);
            }
            if (out->hit_count) out->hit_count[(size_t)fi * NO + o] = (int64_t)nh;
            out->hits_total += (int64_t)nh;
            if (written + (int64_t)nh <= out->hit_cap) {
                hh.resize(nh);
                if (nh) cudaMemcpyAsync(hh.data(), dHits, nh * sizeof(ug_hit), cudaMemcpyDeviceToHost, st);
                if (cudaStreamSynchronize(st) != cudaSuccess) return set_error(UG_ECUDA, "frame_bake: hit copy failed");
                // device append order is scheduling-dependent: sort by (chi, src)
                std::sort(hh.begin(), hh.end(), [](const ug_hit& x, const ug_hit& y) {
                    return x.chi < y.chi || (x.chi == y.chi && x.src < y.src);
                });
                if (nh) memcpy(out->hits + written, hh.data(), nh * sizeof(ug_hit));
                written += (int64_t)nh;
            }
        }
    }
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        std::string m = std::string("frame_bake: ") + cudaGetErrorString(e);
        return set_error(UG_ECUDA, m.c_str());
    }
    if (!want_hits) {
        std::vector<unsigned long long> counts((size_t)NF * NO);
        if (cudaMemcpyAsync(counts.data(), dCount, counts.size() * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return set_error(UG_ECUDA, "frame_bake: count copy failed");
        for (size_t i = 0; i < counts.size(); i++) {
            if (counts[i] > hitCap) return set_error(UG_ECAP, "frame_bake: hit cap overflow (lower the wraps)");
            if (out->hit_count) out->hit_count[i] = (int64_t)counts[i];
            out->hits_total += (int64_t)counts[i];
        }
        if (want_density && (cudaMemcpyAsync(out->density, dDen, bins2 * NF * NO * 4, cudaMemcpyDeviceToHost, st) !=
                                 cudaSuccess ||
                             cudaStreamSynchronize(st) != cudaSuccess))
            return set_error(UG_ECUDA, "frame_bake: density copy failed");
    }
    if (want_hits && out->hits_total > out->hit_cap) return set_error(UG_ECAP, "frame_bake: hit buffer too small");
    return UG_OK;
}

}  // namespace

__global__ void k_fb_maxb(int64_t m, const int32_t* b, int* out) {
    int mx = 2;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        mx = max(mx, b[i]);
    atomicMax(out, mx);
}

// Largest frequency of device-resident dump parameters.
int max_b_device(const int32_t* b, int64_t m, int* out, cudaStream_t st) {
    int* d = nullptr;
    if (cudaMalloc(&d, 4) != cudaSuccess) return set_error(UG_ENOMEM, "frame_bake: device allocation failed");
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaMemsetAsync(d, 0, 4, st);
    k_fb_maxb<<<nsm * 4, 256, 0, st>>>(m, b, d);
    cudaError_t e = cudaMemcpyAsync(out, d, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    return e == cudaSuccess ? UG_OK : set_error(UG_ECUDA, "frame_bake: reduction failed");
}

// Frames of the accepted paths of a packer universe, straight from the device
// (the dump -> frame_bake pipeline without a CSV or host round trip).
int frames_from_params(const ug_frames_cfg* cfg, int n, int nw, int bMax, const double* dA2, const double* dA,
                       const int32_t* dBi, const double* dF, ug_frames_out* out, cudaStream_t st) {
    int rc = check_cfg(cfg, out, n);
    if (rc) return rc;
    DevBuf buf;
    double* dB = buf.get<double>((size_t)n * 2 * nw);
    if (!dB) return set_error(UG_ENOMEM, "frame_bake: device allocation failed");
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    k_fb_from_params<<<nsm * 8, 256, 0, st>>>((int64_t)n * 2 * nw, dBi, dB);
    std::vector<ObsPath> obs(cfg->n_obs);
    for (int o = 0; o < cfg->n_obs; o++) {
        if (cfg->obs_type[o] != 0) continue;
        const int p = cfg->obs_path[o];
        ObsPath& q = obs[o];
        q.a2.resize(2);
        q.a.resize(2 * nw);
        q.b.resize(2 * nw);
        q.f.resize(2 * nw);
        std::vector<int32_t> bi(2 * nw);
        if (cudaMemcpyAsync(q.a2.data(), dA2 + (size_t)p * 2, 16, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(q.a.data(), dA + (size_t)p * 2 * nw, 16 * nw, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(bi.data(), dBi + (size_t)p * 2 * nw, 8 * nw, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(q.f.data(), dF + (size_t)p * 2 * nw, 16 * nw, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return set_error(UG_ECUDA, "frame_bake: observer copy failed");
        for (int j = 0; j < 2 * nw; j++) q.b[j] = bi[j];
    }
    return bake_device(cfg, n, nw, bMax, dA2, dA, dB, dF, obs, out, st);
}

}  // namespace ug

using namespace ug;

extern "C" int ug_frame_bake(const ug_frames_cfg* cfg, int32_t n, int32_t nw, const double* a2,
                             const double* a, const double* b, const double* f, ug_frames_out* out) {
    if (nw < 1 || !a2 || !a || !b || !f) return set_error(UG_EINVAL, "frame_bake: bad arguments");
    int rc = check_cfg(cfg, out, n);
    if (rc) return rc;
    int bMax = 2;
    for (size_t i = 0; i < (size_t)n * 2 * nw; i++) bMax = std::max(bMax, (int)b[i]);
    DevBuf buf;
    const size_t m = (size_t)n * 2 * nw;
    double* dA2 = buf.get<double>((size_t)n * 2);
    double* dA = buf.get<double>(m);
    double* dB = buf.get<double>(m);
    double* dF = buf.get<double>(m);
    if (!dA2 || !dA || !dB || !dF) return set_error(UG_ENOMEM, "frame_bake: device allocation failed");
    // the library's own stream for this call (host buffers in, host buffers out)
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
        return set_error(UG_ECUDA, "frame_bake: stream creation failed");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    cudaMemcpyAsync(dA2, a2, (size_t)n * 2 * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dA, a, m * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dB, b, m * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dF, f, m * 8, cudaMemcpyHostToDevice, st);
    std::vector<ObsPath> obs(cfg->n_obs);
    for (int o = 0; o < cfg->n_obs; o++) {
        if (cfg->obs_type[o] != 0) continue;
        const size_t p = (size_t)cfg->obs_path[o];
        obs[o].a2.assign(a2 + p * 2, a2 + p * 2 + 2);
        obs[o].a.assign(a + p * 2 * nw, a + (p + 1) * 2 * nw);
        obs[o].b.assign(b + p * 2 * nw, b + (p + 1) * 2 * nw);
        obs[o].f.assign(f + p * 2 * nw, f + (p + 1) * 2 * nw);
    }
    return bake_device(cfg, n, nw, bMax, dA2, dA, dB, dF, obs, out, st);
}

// ------------------------------------------------------- observer view remap

namespace ug {
namespace {

// The boost of one observer frame, set up on the host with the reference's
// operations in its order (braidlab/frames.py:164-174): cap, static threshold,
// gamma, unit vector, and the two scalar products it forms once.
struct ViewBoost {
    int moving, cheb;
    double bx, by, ux, uy, gamma, gm1, gbx, gby;
};

constexpr double kBetaCap = 0.995;  // FRAME_BETA_CAP (braidlab/frames.py:37)

ViewBoost view_boost(double beta_x, double beta_y, int mode, int cheb) {
    ViewBoost v{};
    v.cheb = cheb != 0;
    if (mode != UG_VIEW_MOVING) return v;
    double bx = beta_x, by = beta_y;
    double bm = std::hypot(bx, by);
    if (bm > kBetaCap) {
        const double s = kBetaCap / bm;
        bx *= s;
        by *= s;
        bm = kBetaCap;
    }
    if (bm <= 1e-6) return v;
    v.moving = 1;
    v.gamma = 1.0 / std::sqrt(1.0 - std::pow(bm, 2.0));
    v.ux = bx / bm;
    v.uy = by / bm;
    v.bx = bx;
    v.by = by;
    v.gbx = v.gamma * bx;
    v.gby = v.gamma * by;
    v.gm1 = v.gamma - 1.0;
    return v;
}

// One thread per hit, FP64, every product and sum rounded on its own (no
// contraction) in the order of braidlab/frames.py:175-188.
__global__ void k_apparent(const ug_hit* __restrict__ hits, int64_t n, ViewBoost v, double* __restrict__ ax,
                           double* __restrict__ ay, double* __restrict__ ld) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const ug_hit h = hits[i];
        const double dx = h.dx, dy = h.dy;
        if (!v.moving) {
            ax[i] = dx;
            ay[i] = dy;
            ld[i] = 0.0;
            continue;
        }
        const double eucl = hypot(dx, dy);
        const bool ok = eucl > 0.0;
        const double nx = ok ? dx / eucl : 0.0, ny = ok ? dy / eucl : 0.0;
        const double bdotn = __dadd_rn(__dmul_rn(v.bx, nx), __dmul_rn(v.by, ny));
        const double udotn = __dadd_rn(__dmul_rn(v.ux, nx), __dmul_rn(v.uy, ny));
        const double dfac = __dmul_rn(v.gamma, __dadd_rn(1.0, bdotn));
        const double gu = __dmul_rn(v.gm1, udotn);
        const double apx = __dadd_rn(__dadd_rn(nx, v.gbx), __dmul_rn(gu, v.ux)) / dfac;
        const double apy = __dadd_rn(__dadd_rn(ny, v.gby), __dmul_rn(gu, v.uy)) / dfac;
        const double chi = h.chi;
        const double norm = v.cheb ? fmax(fabs(apx), fabs(apy)) : 1.0;
        ax[i] = ok ? __dmul_rn(apx, chi) / norm : dx;
        ay[i] = ok ? __dmul_rn(apy, chi) / norm : dy;
        ld[i] = ok ? log(dfac) : 0.0;
    }
}

int check_view(int64_t n, int32_t mode) {
    if (n < 0) return set_error(UG_EINVAL, "apparent_positions: negative hit count");
    if (mode != UG_VIEW_STATIC && mode != UG_VIEW_MOVING)
        return set_error(UG_EINVAL, "apparent_positions: mode must be static|moving");
    return UG_OK;
}

}  // namespace
}  // namespace ug

extern "C" int ug_apparent_positions_async(const ug_hit* d_hits, int64_t n, double beta_x, double beta_y,
                                           int32_t mode, int32_t cheb, double* d_ax, double* d_ay,
                                           double* d_ln_dopp, void* stream) {
    int rc = check_view(n, mode);
    if (rc || n == 0) return rc;
    if (!d_hits || !d_ax || !d_ay || !d_ln_dopp) return set_error(UG_EINVAL, "apparent_positions: null buffer");
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return set_error(UG_ECUDA, "apparent_positions: no CUDA device");
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)nsm * 8);
    k_apparent<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(d_hits, n, view_boost(beta_x, beta_y, mode, cheb),
                                                                   d_ax, d_ay, d_ln_dopp);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(UG_ECUDA, cudaGetErrorString(e));
    return UG_OK;
}

extern "C" int ug_apparent_positions(const ug_hit* hits, int64_t n, double beta_x, double beta_y, int32_t mode,
                                     int32_t cheb, double* ax, double* ay, double* ln_dopp) {
    int rc = check_view(n, mode);
    if (rc || n == 0) return rc;
    if (!hits || !ax || !ay || !ln_dopp) return set_error(UG_EINVAL, "apparent_positions: null buffer");
    DevBuf buf;
    ug_hit* dH = buf.get<ug_hit>((size_t)n);
    double* dO = buf.get<double>((size_t)n * 3);
    if (!dH || !dO) return set_error(UG_ENOMEM, "apparent_positions: device allocation failed");
    if (cudaMemcpy(dH, hits, (size_t)n * sizeof(ug_hit), cudaMemcpyHostToDevice) != cudaSuccess)
        return set_error(UG_ECUDA, "apparent_positions: hit copy failed");
    rc = ug_apparent_positions_async(dH, n, beta_x, beta_y, mode, cheb, dO, dO + n, dO + 2 * n, nullptr);
    if (rc) return rc;
    if (cudaMemcpy(ax, dO, (size_t)n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(ay, dO + n, (size_t)n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(ln_dopp, dO + 2 * n, (size_t)n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_error(UG_ECUDA, "apparent_positions: result copy failed");
    return UG_OK;
}
