// Genetic-algorithm variation and selection on the GPU, so that a generation
// (offspring -> simulation -> features -> scores -> survivors) never leaves
// the device.
//
// The reference runs these steps on the host between simulator calls:
// DEAP's varOr / eaMuPlusLambda (GUI/DEAP_helper.py:126-271) and bluepyopt's
// DEAPOptimisation with a multi-objective selector
// (Figures/Figure4_DEAP/optimize_parameters_genetic_alg.py:49).  Restated
// here from the published operators:
//   * binary tournament on (front rank ascending, crowding descending);
//   * bounded simulated binary crossover (Deb & Agrawal 1995, in the bounded
//     form of Deb's NSGA-II code) and bounded polynomial mutation (Deb &
//     Goyal 1996), genes in [low, up];
//   * (mu + lambda) truncation on a scalar score, or NSGA-II's
//     non-dominated sorting with crowding distance (Deb, Pratap, Agarwal &
//     Meyarivan 2002) on a vector of objectives, all minimised.
//
// Random numbers are counter based: draw d of child c in generation g is
// SplitMix64 (Steele, Lea & Flood 2014) of a key made from the seed, g, c and
// d, so any child is reproducible on its own and the host restatement
// replays the same stream bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

namespace ngpu {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// the generation's stream key
__host__ __device__ __forceinline__ uint64_t ga_key(uint64_t seed, uint64_t generation) {
    return splitmix64(seed ^ splitmix64(generation));
}

// draw d (< 2^20) of child c: 64 random bits
__device__ __forceinline__ uint64_t ga_bits(uint64_t key, uint64_t child, uint32_t d) {
    return splitmix64(key ^ splitmix64((child << 20) | d));
}

// uniform in [0, 1) with 53 random bits
__device__ __forceinline__ double ga_uniform(uint64_t key, uint64_t child, uint32_t d) {
    return (double)(ga_bits(key, child, d) >> 11) * 0x1.0p-53;
}

// uniform integer in [0, n): the high 32 bits scaled by n (multiply-shift)
__device__ __forceinline__ int ga_index(uint64_t key, uint64_t child, uint32_t d, int n) {
    return (int)(((ga_bits(key, child, d) >> 32) * (uint64_t)n) >> 32);
}

// draw layout of one child: 4 tournament picks, mate, which child of the
// pair; then 5 per gene (crossover?, crossover spread, swap?, mutate?,
// mutation spread)
constexpr uint32_t kGaDrawsFixed = 6;
constexpr uint32_t kGaDrawsPerGene = 5;

struct GaVariation {
    const double* pop;       // [mu][n_genes]
    const int32_t* rank;     // [mu] front rank (lower is better)
    const double* crowd;     // [mu] crowding (higher is better among equal ranks)
    int mu, n_genes, n_kids;
    double low, up, eta_c, eta_m, cx_prob, p_mut;
    uint64_t key;
    double* kids;            // [n_kids][n_genes]
};

__device__ __forceinline__ int ga_tournament(const GaVariation& a, int i, int j) {
    if (a.rank[j] < a.rank[i]) return j;
    if (a.rank[j] == a.rank[i] && a.crowd[j] > a.crowd[i]) return j;
    return i;   // ties: the first pick
}

// spread factor of bounded SBX for one side: beta is 1 + 2 (distance from
// the nearer parent to the bound) / (parent distance)
__device__ __forceinline__ double sbx_beta_q(double beta, double u, double eta) {
    const double alpha = 2.0 - pow(beta, -(eta + 1.0));
    if (u <= 1.0 / alpha) return pow(u * alpha, 1.0 / (eta + 1.0));
    return pow(1.0 / (2.0 - u * alpha), 1.0 / (eta + 1.0));
}

__global__ void __launch_bounds__(128) k_ga_offspring(const GaVariation a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n_kids) return;
    const uint64_t key = a.key, ch = (uint64_t)c;
    const int p1 = ga_tournament(a, ga_index(key, ch, 0, a.mu), ga_index(key, ch, 1, a.mu));
    const int p2 = ga_tournament(a, ga_index(key, ch, 2, a.mu), ga_index(key, ch, 3, a.mu));
    const bool mate = ga_uniform(key, ch, 4) < a.cx_prob;
    const bool first = ga_uniform(key, ch, 5) < 0.5;
    const double* x = a.pop + (size_t)p1 * a.n_genes;
    const double* y = a.pop + (size_t)p2 * a.n_genes;
    double* out = a.kids + (size_t)c * a.n_genes;
    const double lo = a.low, hi = a.up, span = hi - lo;
    for (int g = 0; g < a.n_genes; ++g) {
        const uint32_t d = kGaDrawsFixed + kGaDrawsPerGene * (uint32_t)g;
        double v = x[g];
        if (mate) {
            // bounded SBX of the pair (x[g], y[g]); the child keeps x[g] where no crossover happens
            const double u_do = ga_uniform(key, ch, d), u = ga_uniform(key, ch, d + 1);
            const double u_sw = ga_uniform(key, ch, d + 2);
            const double a1 = x[g], b1 = y[g];
            if (u_do < 0.5 && fabs(a1 - b1) > 1e-14) {
                const double x1 = fmin(a1, b1), x2 = fmax(a1, b1), dx = x2 - x1;
                const double y1 = fmin(fmax(0.5 * (x1 + x2 - sbx_beta_q(1.0 + 2.0 * (x1 - lo) / dx, u, a.eta_c) * dx), lo), hi);
                const double y2 = fmin(fmax(0.5 * (x1 + x2 + sbx_beta_q(1.0 + 2.0 * (hi - x2) / dx, u, a.eta_c) * dx), lo), hi);
                const bool swap = u_sw < 0.5;
                // the pair's children are (y1, y2), or (y2, y1) when swapped; this child is the first or the second
                v = (first != swap) ? y1 : y2;
            } else if (!first) {
                v = b1;
            }
        }
        // bounded polynomial mutation
        if (ga_uniform(key, ch, d + 3) < a.p_mut) {
            const double r = ga_uniform(key, ch, d + 4);
            const double d1 = (v - lo) / span, d2 = (hi - v) / span, mp = 1.0 / (a.eta_m + 1.0);
            double dq;
            if (r < 0.5) {
                const double val = 2.0 * r + (1.0 - 2.0 * r) * pow(1.0 - d1, a.eta_m + 1.0);
                dq = pow(val, mp) - 1.0;
            } else {
                const double val = 2.0 * (1.0 - r) + 2.0 * (r - 0.5) * pow(1.0 - d2, a.eta_m + 1.0);
                dq = 1.0 - pow(val, mp);
            }
            v = fmin(fmax(v + dq * span, lo), hi);
        }
        out[g] = v;
    }
}

// --------------------------------------------------------------- sorting
// Total order of doubles as unsigned keys (NaN after +inf).
__host__ __device__ __forceinline__ uint64_t ga_order_key(double x) {
    if (x != x) return 0xFFFFFFFFFFFFFFFEull;
    uint64_t b;
    memcpy(&b, &x, 8);
    if (x == 0.0) b = 0;                       // -0 and +0 alike
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

struct GaSortSlice {
    uint64_t* k1;
    uint64_t* k2;
    uint32_t* idx;
};

__device__ __forceinline__ bool ga_less(const GaSortSlice& s, uint32_t a, uint32_t b) {
    if (s.k1[a] != s.k1[b]) return s.k1[a] < s.k1[b];
    if (s.k2[a] != s.k2[b]) return s.k2[a] < s.k2[b];
    return s.idx[a] < s.idx[b];
}

// Bitonic sort of n2 (a power of two) entries by (k1, k2, idx), ascending,
// by one CTA over global memory; the barrier after each stage orders the
// block's global writes.
__device__ void ga_bitonic(const GaSortSlice& s, uint32_t n2) {
    for (uint32_t k = 2; k <= n2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const bool asc = (i & k) == 0;
                    if (ga_less(s, l, i) == asc) {
                        const uint64_t a1 = s.k1[i], a2 = s.k2[i];
                        const uint32_t ai = s.idx[i];
                        s.k1[i] = s.k1[l];
                        s.k2[i] = s.k2[l];
                        s.idx[i] = s.idx[l];
                        s.k1[l] = a1;
                        s.k2[l] = a2;
                        s.idx[l] = ai;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// keys of (mu + lambda) truncation: the score, then the index
__global__ void k_ga_truncation_keys(const double* score, int n, uint32_t n2, GaSortSlice s) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
        const bool in = i < (uint32_t)n;
        s.k1[i] = in ? ga_order_key(score[i]) : ~0ull;
        s.k2[i] = 0;
        s.idx[i] = i;
    }
}

__global__ void __launch_bounds__(1024) k_ga_sort(GaSortSlice s, uint32_t n2) { ga_bitonic(s, n2); }

__global__ void k_ga_take(const uint32_t* sorted_idx, int mu, int32_t* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < mu; i += gridDim.x * blockDim.x) out[i] = (int32_t)sorted_idx[i];
}

// ------------------------------------------------------------- NSGA-II
// objectives [n][m] -> [m][n], NaN as +inf (worst)
__global__ void k_ga_transpose(const double* obj, int n, int m, double* fT) {
    const size_t total = (size_t)n * m;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t i = t / m, k = t % m;
        const double x = obj[t];
        fT[k * n + i] = x != x ? INFINITY : x;
    }
}

// dom[i][w] bit b: individual j = 32 w + b dominates i (no worse in every
// objective, better in one).  Block: 256 individuals i against the 32 of
// word w, whose objectives are staged in shared memory.
constexpr int kGaDomThreads = 256;

__global__ void __launch_bounds__(kGaDomThreads) k_ga_dominance(const double* fT, int n, int m, int W, uint32_t* dom) {
    extern __shared__ double fj[];   // [m][32]
    const int w = blockIdx.y, j0 = 32 * w;
    for (int t = threadIdx.x; t < m * 32; t += blockDim.x) {
        const int k = t >> 5, jj = t & 31;
        fj[t] = j0 + jj < n ? fT[(size_t)k * n + j0 + jj] : INFINITY;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int valid = n - j0;
    uint32_t le = valid >= 32 ? 0xFFFFFFFFu : ((1u << valid) - 1u), lt = 0;
    for (int k = 0; k < m && le; ++k) {
        const double fi = fT[(size_t)k * n + i];
        const double* row = fj + k * 32;
        uint32_t lem = 0, ltm = 0;
#pragma unroll
        for (int jj = 0; jj < 32; ++jj) {
            lem |= (uint32_t)(row[jj] <= fi) << jj;
            ltm |= (uint32_t)(row[jj] < fi) << jj;
        }
        le &= lem;
        lt |= ltm;
    }
    dom[(size_t)i * W + w] = le & lt;
}

// Front ranks by peeling: front r holds the individuals no remaining one
// dominates.  One CTA; every front is non-empty (dominance is a strict
// partial order), so at most n rounds.
constexpr int kGaMaxWords = 1024;   // n <= 32768

__global__ void __launch_bounds__(1024) k_ga_fronts(const uint32_t* dom, int n, int W, int32_t* rank, int32_t* n_fronts) {
    __shared__ uint32_t R[kGaMaxWords], NF[kGaMaxWords];
    __shared__ int remaining;
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        const int valid = n - 32 * w;
        R[w] = valid >= 32 ? 0xFFFFFFFFu : ((1u << valid) - 1u);
    }
    if (threadIdx.x == 0) remaining = n;
    __syncthreads();
    int front = 0;
    for (; front < n && remaining > 0; ++front) {
        for (int w = threadIdx.x; w < W; w += blockDim.x) NF[w] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            if (!((R[i >> 5] >> (i & 31)) & 1u)) continue;
            const uint32_t* row = dom + (size_t)i * W;
            bool dominated = false;
            for (int w = 0; w < W; ++w) {
                if (row[w] & R[w]) {
                    dominated = true;
                    break;
                }
            }
            if (!dominated) {
                atomicOr(&NF[i >> 5], 1u << (i & 31));
                rank[i] = front;
            }
        }
        __syncthreads();
        int removed = 0;
        for (int w = threadIdx.x; w < W; w += blockDim.x) {
            R[w] &= ~NF[w];
            removed += __popc(NF[w]);
        }
        if (removed) atomicSub(&remaining, removed);
        __syncthreads();
    }
    // unreachable with every front non-empty; kept so that a rank is always a valid index
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if ((R[i >> 5] >> (i & 31)) & 1u) rank[i] = min(front, n - 1);
    if (threadIdx.x == 0) *n_fronts = remaining == 0 ? front : -1;
}

// Crowding distance, one CTA per objective k: sort by (rank, f_k, index);
// the first and last of each front get +inf, the others (f_next - f_prev) /
// (f_last - f_first) of their front (0 where the front is flat in f_k).
struct GaCrowdArgs {
    const double* fT;        // [m][n]
    const int32_t* rank;     // [n]
    int n, m;
    uint32_t n2;
    uint64_t* k1;            // [m][n2] workspace
    uint64_t* k2;
    uint32_t* idx;
    int32_t* start;          // [m][n] first sorted position of each rank
    int32_t* end;
    double* contrib;         // [m][n]
};

__global__ void __launch_bounds__(1024) k_ga_crowding(const GaCrowdArgs a) {
    const int k = blockIdx.x;
    const double* f = a.fT + (size_t)k * a.n;
    GaSortSlice s{a.k1 + (size_t)k * a.n2, a.k2 + (size_t)k * a.n2, a.idx + (size_t)k * a.n2};
    int32_t* st = a.start + (size_t)k * a.n;
    int32_t* en = a.end + (size_t)k * a.n;
    for (uint32_t i = threadIdx.x; i < a.n2; i += blockDim.x) {
        const bool in = i < (uint32_t)a.n;
        s.k1[i] = in ? (uint64_t)a.rank[i] : ~0ull;
        s.k2[i] = in ? ga_order_key(f[i]) : ~0ull;
        s.idx[i] = i;
    }
    __syncthreads();
    ga_bitonic(s, a.n2);
    for (int p = threadIdx.x; p < a.n; p += blockDim.x) {
        const uint64_t r = s.k1[p];
        if (p == 0 || s.k1[p - 1] != r) st[r] = p;
        if (p == a.n - 1 || s.k1[p + 1] != r) en[r] = p;
    }
    __syncthreads();
    double* out = a.contrib + (size_t)k * a.n;
    for (int p = threadIdx.x; p < a.n; p += blockDim.x) {
        const uint64_t r = s.k1[p];
        const int p0 = st[r], p1 = en[r];
        double c;
        if (p == p0 || p == p1) {
            c = INFINITY;
        } else {
            const double lo = f[s.idx[p0]], hi = f[s.idx[p1]];
            c = hi == lo ? 0.0 : (f[s.idx[p + 1]] - f[s.idx[p - 1]]) / (hi - lo);
        }
        out[s.idx[p]] = c;
    }
}

// crowd[i] = sum over objectives in order; then the survivor keys (rank,
// -crowd, index)
__global__ void k_ga_crowd_sum(const double* contrib, const int32_t* rank, int n, int m, uint32_t n2, double* crowd,
                               GaSortSlice s) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
        if (i < (uint32_t)n) {
            double c = 0.0;
            for (int k = 0; k < m; ++k) c += contrib[(size_t)k * n + i];
            crowd[i] = c;
            s.k1[i] = (uint64_t)rank[i];
            s.k2[i] = ga_order_key(-c);
        } else {
            s.k1[i] = ~0ull;
            s.k2[i] = ~0ull;
        }
        s.idx[i] = i;
    }
}

}  // namespace ngpu
