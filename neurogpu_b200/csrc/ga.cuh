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
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

namespace ngpu {

namespace cg = cooperative_groups;

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

// Segmented bitonic sort: `count` independent segments of n2 entries (a
// power of two) each, ascending by (k1, k2, idx).  Strides below the tile
// (kGaSortTile entries, one CTA) run in shared memory -- the whole network
// up to the tile size at first, then the tail of every later merge; strides
// of a tile or more run as grid-wide stages, one launch each, every thread
// one compare-exchange.  The direction of a pair follows its position in its
// segment, so segments never mix.
constexpr uint32_t kGaSortTile = 2048;
constexpr int kGaSortThreads = 1024;

__device__ __forceinline__ void ga_cmpswap(uint64_t* k1, uint64_t* k2, uint32_t* ix, size_t i, size_t l, bool asc) {
    const bool less_li = k1[l] != k1[i] ? k1[l] < k1[i] : (k2[l] != k2[i] ? k2[l] < k2[i] : ix[l] < ix[i]);
    if (less_li == asc) {
        const uint64_t a1 = k1[i], a2 = k2[i];
        const uint32_t ai = ix[i];
        k1[i] = k1[l];
        k2[i] = k2[l];
        ix[i] = ix[l];
        k1[l] = a1;
        k2[l] = a2;
        ix[l] = ai;
    }
}

// one tile per CTA: k_merge == 0 sorts the tile (every k up to the tile
// size); otherwise the strides below the tile of merge step k_merge
__global__ void __launch_bounds__(kGaSortThreads) k_ga_sort_tile(GaSortSlice s, uint32_t n2, uint32_t tile,
                                                                 uint32_t k_merge) {
    __shared__ uint64_t k1[kGaSortTile], k2[kGaSortTile];
    __shared__ uint32_t ix[kGaSortTile];
    const size_t base = (size_t)blockIdx.x * tile;
    for (uint32_t t = threadIdx.x; t < tile; t += blockDim.x) {
        k1[t] = s.k1[base + t];
        k2[t] = s.k2[base + t];
        ix[t] = s.idx[base + t];
    }
    __syncthreads();
    const uint32_t pos0 = (uint32_t)(base & (n2 - 1));   // position of the tile in its segment
    const uint32_t k_lo = k_merge ? k_merge : 2, k_hi = k_merge ? k_merge : tile;
    for (uint32_t k = k_lo; k <= k_hi; k <<= 1) {
        for (uint32_t j = (k_merge ? tile : k) >> 1; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < tile; t += blockDim.x) {
                const uint32_t l = t ^ j;
                if (l > t) ga_cmpswap(k1, k2, ix, t, l, ((pos0 + t) & k) == 0);
            }
            __syncthreads();
        }
    }
    for (uint32_t t = threadIdx.x; t < tile; t += blockDim.x) {
        s.k1[base + t] = k1[t];
        s.k2[base + t] = k2[t];
        s.idx[base + t] = ix[t];
    }
}

// one grid-wide stage (k, j) with j >= the tile: pair p -> (i, i + j), bit j of i clear
__global__ void k_ga_sort_stage(GaSortSlice s, size_t total, uint32_t n2, uint32_t k, uint32_t j) {
    const size_t pairs = total >> 1;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < pairs; p += (size_t)gridDim.x * blockDim.x) {
        const size_t i = (p / j) * (2 * (size_t)j) + (p % j);
        ga_cmpswap(s.k1, s.k2, s.idx, i, i + j, ((uint32_t)(i & (n2 - 1)) & k) == 0);
    }
}

// host side: sort `count` segments of n2 entries on a stream; returns the launches issued
inline int ga_sort(const GaSortSlice& s, uint32_t n2, int count, cudaStream_t st) {
    const uint32_t tile = n2 < kGaSortTile ? n2 : kGaSortTile;
    const size_t total = (size_t)n2 * count;
    const unsigned tiles = (unsigned)(total / tile);
    const unsigned grid = (unsigned)std::min<size_t>((total / 2 + 255) / 256, 148 * 16);
    int launches = 1;
    k_ga_sort_tile<<<tiles, kGaSortThreads, 0, st>>>(s, n2, tile, 0);
    for (uint32_t k = 2 * tile; k <= n2; k <<= 1) {
        for (uint32_t j = k >> 1; j >= tile; j >>= 1) {
            k_ga_sort_stage<<<grid, 256, 0, st>>>(s, total, n2, k, j);
            ++launches;
        }
        k_ga_sort_tile<<<tiles, kGaSortThreads, 0, st>>>(s, n2, tile, k);
        ++launches;
    }
    return launches;
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
// dominates.  A cooperative grid: each round, every CTA stages the remaining
// set R in shared memory and tests its share of individuals against it
// (dominance rows are read until a remaining dominator turns up, so a
// round's traffic is spread over the grid); new front members are or-ed
// into NF; after a grid barrier R loses NF.  Every front is non-empty
// (dominance is a strict partial order), so at most n rounds.  R, NF and
// the count are written by other CTAs: they are read through L2 (__ldcg).
constexpr int kGaMaxWords = 1024;   // n <= 32768
constexpr int kGaFrontThreads = 256;

struct GaFrontArgs {
    const uint32_t* dom;     // [n][W]
    int n, W;
    int32_t* rank;           // [n]
    uint32_t* R;             // [W] remaining
    uint32_t* NF;            // [W] this round's front
    int* remaining;
    int32_t* n_fronts;
};

__global__ void __launch_bounds__(kGaFrontThreads) k_ga_fronts(const GaFrontArgs a) {
    cg::grid_group grid = cg::this_grid();
    __shared__ uint32_t Rs[kGaMaxWords];
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    for (int w = gtid; w < a.W; w += gstride) {
        const int valid = a.n - 32 * w;
        a.R[w] = valid >= 32 ? 0xFFFFFFFFu : ((1u << valid) - 1u);
        a.NF[w] = 0;
    }
    if (gtid == 0) *a.remaining = a.n;
    grid.sync();
    int front = 0;
    for (; front < a.n; ++front) {
        if (__ldcg(a.remaining) == 0) break;    // the same value in every thread: read after the barrier
        for (int w = threadIdx.x; w < a.W; w += blockDim.x) Rs[w] = __ldcg(a.R + w);
        __syncthreads();
        for (int i = gtid; i < a.n; i += gstride) {
            if (!((Rs[i >> 5] >> (i & 31)) & 1u)) continue;
            const uint32_t* row = a.dom + (size_t)i * a.W;
            bool dominated = false;
            for (int w = 0; w < a.W; ++w) {
                if (row[w] & Rs[w]) {
                    dominated = true;
                    break;
                }
            }
            if (!dominated) {
                atomicOr(a.NF + (i >> 5), 1u << (i & 31));
                a.rank[i] = front;
            }
        }
        grid.sync();
        for (int w = gtid; w < a.W; w += gstride) {
            const uint32_t nf = __ldcg(a.NF + w);
            if (nf) {
                a.R[w] = __ldcg(a.R + w) & ~nf;
                a.NF[w] = 0;
                atomicSub(a.remaining, __popc(nf));
            }
        }
        grid.sync();
    }
    // unreachable with every front non-empty; kept so that a rank is always a valid index
    for (int i = gtid; i < a.n; i += gstride)
        if ((__ldcg(a.R + (i >> 5)) >> (i & 31)) & 1u) a.rank[i] = min(front, a.n - 1);
    if (gtid == 0) *a.n_fronts = __ldcg(a.remaining) == 0 ? front : -1;
}

// Crowding distance per objective k (one sorted segment each): sort by
// (rank, f_k, index); the first and last of each front get +inf, the others
// (f_next - f_prev) / (f_last - f_first) of their front (0 where the front is
// flat in f_k).
struct GaCrowdArgs {
    const double* fT;        // [m][n]
    const int32_t* rank;     // [n]
    int n, m;
    uint32_t n2;
    GaSortSlice s;           // [m][n2]
    int32_t* start;          // [m][n] first sorted position of each rank
    int32_t* end;
    double* contrib;         // [m][n]
};

__global__ void k_ga_crowd_keys(const GaCrowdArgs a) {
    const size_t total = (size_t)a.m * a.n2;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t k = t / a.n2;
        const uint32_t i = (uint32_t)(t % a.n2);
        const bool in = i < (uint32_t)a.n;
        a.s.k1[t] = in ? (uint64_t)a.rank[i] : ~0ull;
        a.s.k2[t] = in ? ga_order_key(a.fT[k * a.n + i]) : ~0ull;
        a.s.idx[t] = i;
    }
}

__global__ void k_ga_crowd_bounds(const GaCrowdArgs a) {
    const size_t total = (size_t)a.m * a.n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t k = t / a.n;
        const int p = (int)(t % a.n);
        const uint64_t* k1 = a.s.k1 + k * a.n2;
        const uint64_t r = k1[p];
        if (p == 0 || k1[p - 1] != r) a.start[k * a.n + r] = p;
        if (p == a.n - 1 || k1[p + 1] != r) a.end[k * a.n + r] = p;
    }
}

__global__ void k_ga_crowd_contrib(const GaCrowdArgs a) {
    const size_t total = (size_t)a.m * a.n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t k = t / a.n;
        const int p = (int)(t % a.n);
        const uint64_t* k1 = a.s.k1 + k * a.n2;
        const uint32_t* ix = a.s.idx + k * a.n2;
        const double* f = a.fT + k * a.n;
        const uint64_t r = k1[p];
        const int p0 = a.start[k * a.n + r], p1 = a.end[k * a.n + r];
        double c;
        if (p == p0 || p == p1) {
            c = INFINITY;
        } else {
            const double lo = f[ix[p0]], hi = f[ix[p1]];
            c = hi == lo ? 0.0 : (f[ix[p + 1]] - f[ix[p - 1]]) / (hi - lo);
        }
        a.contrib[k * a.n + ix[p]] = c;
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
