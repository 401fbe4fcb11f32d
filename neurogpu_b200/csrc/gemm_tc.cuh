// BF16 tensor-core GEMM for the surrogate network (tcgen05, sm_100a).
//
//   D[M][N] = A[M][K] . B[N][K]^T     (A, B bf16, both K-major; D fp32 in TMEM)
//
// One CTA of 128 threads computes a 128 x BN tile over a range of K (all of
// K, or one slice of it for the split-K epilogue).  K advances in tiles of
// 64 through an S-stage shared-memory ring (S = 4, 3 for BN = 256): all
// threads copy tile k + S - 1 into its stage with cp.async (rows past M read
// as zeros) while the tensor cores work on tiles k .. k + S - 2; one thread
// issues four tcgen05.mma (K = 16 each) per tile and commits them to that
// stage's mbarrier, which the copy into the stage waits on before
// overwriting it.  The accumulator lives in tensor memory (BN fp32 columns x
// 128 lanes); after the last commit each warp reads its 32 lanes with
// tcgen05.ld, 16 columns at a time, and stages them through shared memory
// (the ring, free by then) so that row-major outputs are written with
// coalesced stores: a warp store covers two rows of 16 columns.
//
// Shared-memory operand layout (no swizzle, K-major canonical layout): an
// 8-row x 16-byte core matrix is 128 contiguous bytes; core matrices along K
// are LBO = 128 bytes apart, blocks of 8 rows SBO = 8 x 128 = 1024 bytes
// apart, so one 64-wide K tile of 128 rows is 16 KB.  Descriptor fields
// (start >> 4, LBO >> 4 at bit 16, SBO >> 4 at bit 32, version 1 at bit 46,
// swizzle 0 at bit 61) and the kind::f16 instruction descriptor (F32
// accumulator, BF16 A and B, K-major both, N >> 3 at bit 17, M >> 4 at
// bit 24) follow the PTX ISA's tcgen05 matrix and instruction descriptors.
//
// Every wait is bounded: past the limit the kernel records an error in
// *err, skips the epilogue and still frees its tensor memory.
//
// k_gemm_bf16_tma below is the TMA-fed, warp-specialised form with
// 128-byte-swizzled operands; the host runs it where it can build the tensor
// maps, and this cp.async kernel otherwise.  k_gemm_bf16_tma_persistent is
// its persistent form (one CTA per SM, two accumulators in tensor memory)
// for GEMMs of more than two tiles per SM.
#pragma once
#include <cuda.h>  // CUtensorMap
#include <cuda_bf16.h>
#include <stdint.h>

namespace ngpu {

constexpr int kGemmThreads = 128;
// The TMA kernel's CTA: one producer thread and one MMA thread during the
// main loop, then all 16 warps in the epilogue (four per 32-lane quarter of
// tensor memory, each on its own column slice).
constexpr int kTmaThreads = 512;
constexpr int kGemmBM = 128;
constexpr int kGemmBK = 64;
constexpr uint32_t kSpinLimit = 1u << 26;

enum GemmEpilogue : int {
    kEpiStore = 0,      // out_f32[m][n] = D
    kEpiBiasGelu = 1,   // z = D + bias[n]: out_f32 = z, out_bf16 = gelu(z), out_bf16_t[n][m] = gelu(z)
    kEpiBias = 2,       // out_f32[m][n] = D + bias[n]
    kEpiGeluGrad = 3,   // dz = D * gelu'(zin[m][n]): out_bf16 = dz, out_bf16_t[n][m] = dz
    kEpiSplitAdd = 4,   // out_f32[m][n] += D over this CTA's slice of K (split-K; out_f32 zeroed first)
};

struct GemmArgs {
    const __nv_bfloat16* A;  // [M][lda]
    const __nv_bfloat16* B;  // [N][ldb]
    int M, N, K, lda, ldb;
    float* out_f32;          // [M][ldo]
    __nv_bfloat16* out_bf16; // [M][ldo]
    __nv_bfloat16* out_bf16_t;  // [N][ldt]
    int ldo, ldt;
    const float* bias;       // [N]
    const float* zin;        // [M][ldo]
    int* err;
    int kt_split;            // 64-wide K tiles per CTA; CTA z takes tiles [z kt_split, (z+1) kt_split)
};

// The tensor-core unit's tanh (tanh.approx.f32, one instruction; relative
// error ~5e-4, below the bf16 rounding of the outputs it feeds).
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu_tanh(float z) {
    const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
    return 0.5f * z * (1.0f + tanh_fast(u));
}
__device__ __forceinline__ float gelu_tanh_grad(float z) {
    const float z2 = z * z;
    const float u = 0.7978845608028654f * (z + 0.044715f * z2 * z);
    const float t = tanh_fast(u);
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * z2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    const uint64_t lbo = 128 >> 4, sbo = 1024 >> 4;
    return (uint64_t)((saddr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

template <int BN>
__device__ __forceinline__ constexpr uint32_t umma_idesc() {
    return (1u << 4)                      // D: F32
           | (1u << 7) | (1u << 10)       // A, B: BF16
           | ((uint32_t)(BN >> 3) << 17)  // N
           | ((uint32_t)(kGemmBM >> 4) << 24);  // M = 128
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// true when the phase completed, false after kSpinLimit polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    const int n = valid ? 16 : 0;  // 0: fill with zeros
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(n) : "memory");
}

// Copy one 64-wide K tile of `rows` rows (row r of the tile at src + r * ld)
// into the core-matrix layout at dst; rows >= rows_valid read as zeros.
template <int ROWS>
__device__ __forceinline__ void load_tile(uint32_t dst, const __nv_bfloat16* src, int ld, int rows_valid) {
    constexpr int kVec = ROWS * (kGemmBK / 8);  // 16-byte vectors
#pragma unroll
    for (int v = threadIdx.x; v < kVec; v += kGemmThreads) {
        const int row = v >> 3, kg = v & 7;
        const uint32_t off = (uint32_t)((row >> 3) * 1024 + kg * 128 + (row & 7) * 16);
        const bool ok = row < rows_valid;
        const __nv_bfloat16* p = src + (size_t)(ok ? row : 0) * ld + kg * 8;
        cp_async16(dst + off, p, ok);
    }
}

// Ring depth: four stages (three for the 256-wide tile, whose stage is 48 KB).
template <int BN>
__host__ __device__ constexpr int gemm_stages() {
    return BN >= 256 ? 3 : 4;
}

template <int BN>
struct GemmSmem {
    static constexpr int kStages = gemm_stages<BN>();
    alignas(1024) unsigned char a[kStages][kGemmBM * kGemmBK * 2];
    alignas(1024) unsigned char b[kStages][BN * kGemmBK * 2];
    alignas(8) uint64_t bar[kStages];
    uint32_t tmem;
};

// Epilogue staging: per warp 32 rows x 16 columns of fp32, row stride 17
// (conflict-free column writes), inside the ring once the MMAs are done.
constexpr int kStageStride = 17;
static_assert(kGemmBM * kGemmBK * 2 >= 4 * 32 * kStageStride * 4, "staging fits in the first A stage");

// One output element of the epilogue: accumulator value *sp of row m,
// column n (o = m * ldo + n); the bf16 epilogues leave their rounded value in
// *sp for the transposed copy.
template <int EPI>
__device__ __forceinline__ void epi_one(const GemmArgs& g, float* sp, size_t o, int n) {
    const float d = *sp;
    if constexpr (EPI == kEpiStore) {
        g.out_f32[o] = d;
    } else if constexpr (EPI == kEpiBias) {
        g.out_f32[o] = d + g.bias[n];
    } else if constexpr (EPI == kEpiSplitAdd) {
        atomicAdd(g.out_f32 + o, d);
    } else if constexpr (EPI == kEpiBiasGelu) {
        const float z = d + g.bias[n];
        const __nv_bfloat16 h = __float2bfloat16_rn(gelu_tanh(z));
        g.out_f32[o] = z;
        g.out_bf16[o] = h;
        *sp = __bfloat162float(h);
    } else {  // kEpiGeluGrad
        const __nv_bfloat16 h = __float2bfloat16_rn(d * gelu_tanh_grad(g.zin[o]));
        g.out_bf16[o] = h;
        *sp = __bfloat162float(h);
    }
}

// Four consecutive elements (n a multiple of 4, all four inside N) with
// 16-byte f32 and 8-byte bf16 accesses; the caller checked the alignment.
template <int EPI>
__device__ __forceinline__ void epi_vec4(const GemmArgs& g, float* sp, size_t o, int n) {
    static_assert(EPI != kEpiSplitAdd, "split-K atomics go one element per lane");
    float d[4] = {sp[0], sp[1], sp[2], sp[3]};
    if constexpr (EPI == kEpiStore || EPI == kEpiBias) {
        if constexpr (EPI == kEpiBias) {
            const float4 b = *reinterpret_cast<const float4*>(g.bias + n);
            d[0] += b.x, d[1] += b.y, d[2] += b.z, d[3] += b.w;
        }
        *reinterpret_cast<float4*>(g.out_f32 + o) = make_float4(d[0], d[1], d[2], d[3]);
    } else {
        float v[4];
        if constexpr (EPI == kEpiBiasGelu) {
            const float4 b = *reinterpret_cast<const float4*>(g.bias + n);
            const float z[4] = {d[0] + b.x, d[1] + b.y, d[2] + b.z, d[3] + b.w};
            *reinterpret_cast<float4*>(g.out_f32 + o) = make_float4(z[0], z[1], z[2], z[3]);
#pragma unroll
            for (int q = 0; q < 4; ++q) v[q] = gelu_tanh(z[q]);
        } else {  // kEpiGeluGrad
            const float4 z = *reinterpret_cast<const float4*>(g.zin + o);
            v[0] = d[0] * gelu_tanh_grad(z.x), v[1] = d[1] * gelu_tanh_grad(z.y);
            v[2] = d[2] * gelu_tanh_grad(z.z), v[3] = d[3] * gelu_tanh_grad(z.w);
        }
        const __nv_bfloat162 lo = __floats2bfloat162_rn(v[0], v[1]), hi = __floats2bfloat162_rn(v[2], v[3]);
        uint2 pk;
        pk.x = *reinterpret_cast<const uint32_t*>(&lo);
        pk.y = *reinterpret_cast<const uint32_t*>(&hi);
        *reinterpret_cast<uint2*>(g.out_bf16 + o) = pk;
        sp[0] = __low2float(lo), sp[1] = __high2float(lo), sp[2] = __low2float(hi), sp[3] = __high2float(hi);
    }
}

// Epilogue of a 128 x BN tile whose accumulator is in tensor memory at
// `tmem`, by NW warps, the CTA's warps w0 .. w0 + NW - 1: warp w reads the 32
// lanes (rows) of quarter w % 4 (the lanes tcgen05.ld lets it reach) over
// column slice (w - w0) / 4 of the tile, 16 columns at a time, stages them in
// shared memory at `stage` (NW x 32 x kStageStride floats) and writes the
// outputs with coalesced stores (see GemmEpilogue).  Any four consecutive
// warps cover the four quarters, so the group w0 + 4k .. w0 + 4k + 3 takes
// slice k whatever w0 is.  Warps past the last slice have no work.
template <int BN, int EPI, int NW = 4>
__device__ __forceinline__ void gemm_epilogue(const GemmArgs& g, uint32_t tmem, float* stage, int m0, int n0,
                                              int w0 = 0) {
    constexpr int kSlices = (NW / 4) < (BN / 16) ? (NW / 4) : (BN / 16);
    constexpr int kCols = BN / kSlices;  // a multiple of 16
    static_assert(NW % 4 == 0 && kCols % 16 == 0, "epilogue slices");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = warp & 3, slice = (warp - w0) >> 2;
    // 4-wide accesses need rows that start on 16 bytes (f32) and 8 bytes (bf16)
    const uintptr_t al16 = (uintptr_t)g.out_f32 | (uintptr_t)g.bias | (uintptr_t)g.zin;
    const bool vec = g.ldo % 4 == 0 && (al16 & 15) == 0 && ((uintptr_t)g.out_bf16 & 7) == 0;
    if (slice < kSlices) {
        const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16);
        float* stg = stage + (warp - w0) * 32 * kStageStride;
        const int mw = m0 + q * 32;  // this warp's first row
#pragma unroll 1
        for (int c0 = slice * kCols; c0 < (slice + 1) * kCols; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(trow + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 16; ++j) stg[lane * kStageStride + j] = __uint_as_float(r[j]);
            __syncwarp();
            if constexpr (EPI == kEpiSplitAdd) {
                // atomics one element per lane: element e = j * 32 + lane is row e / 16,
                // column e % 16 (a warp's atomics cover 2 rows of 16 columns)
#pragma unroll 4
                for (int j = 0; j < 16; ++j) {
                    const int e = j * 32 + lane, row = e >> 4, col = e & 15;
                    const int m = mw + row, n = n0 + c0 + col;
                    if (m < g.M && n < g.N)
                        epi_one<EPI>(g, stg + row * kStageStride + col, (size_t)m * g.ldo + n, n);
                }
            } else {
                // coalesced pass: group e = j * 32 + lane is row e / 4, columns 4 (e % 4) .. + 3
                // (a warp store covers 8 rows of 16 columns)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int e = j * 32 + lane, row = e >> 2, cg = (e & 3) * 4;
                    const int m = mw + row, n = n0 + c0 + cg;
                    float* sp = stg + row * kStageStride + cg;
                    if (m < g.M && n < g.N) {
                        const size_t o = (size_t)m * g.ldo + n;
                        if (vec && n + 4 <= g.N) {
                            epi_vec4<EPI>(g, sp, o, n);
                        } else {
#pragma unroll
                            for (int k = 0; k < 4; ++k)
                                if (n + k < g.N) epi_one<EPI>(g, sp + k, o + k, n + k);
                        }
                    }
                }
            }
            if constexpr (EPI == kEpiBiasGelu || EPI == kEpiGeluGrad) {
                // the transposed bf16 copy, lane = row: a warp store is 32 consecutive rows
                __syncwarp();
                const int m = mw + lane;
                if (m < g.M) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int n = n0 + c0 + j;
                        if (n < g.N)
                            g.out_bf16_t[(size_t)n * g.ldt + m] = __float2bfloat16_rn(stg[lane * kStageStride + j]);
                    }
                }
            }
            __syncwarp();  // the next chunk overwrites the staging rows
        }
    }
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16_tn(GemmArgs g) {
    static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256, "BN: a multiple of 16 in [32, 256]");
    constexpr int S = gemm_stages<BN>();
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // align the ring to 1024 bytes (descriptor base offset 0)
    GemmSmem<BN>& Sm = *reinterpret_cast<GemmSmem<BN>*>(
        (void*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
    const int warp = threadIdx.x >> 5;
    const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * BN;
    constexpr uint32_t kCols = BN < 32 ? 32 : BN;  // power of two >= 32 for BN in {32, 64, 128, 256}

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&Sm.tmem)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(smem_u32(&Sm.bar[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = Sm.tmem;

    // this CTA's K tiles: [kt0, kt0 + KT) (the host gives every CTA at least one)
    const int kt0 = blockIdx.z * g.kt_split;
    const int KT = min(g.kt_split, g.K / kGemmBK - kt0);
    const int rows_a = min(kGemmBM, g.M - m0), rows_b = min(BN, g.N - n0);
    const __nv_bfloat16* Ab = g.A + (size_t)m0 * g.lda + (size_t)kt0 * kGemmBK;
    const __nv_bfloat16* Bb = g.B + (size_t)n0 * g.ldb + (size_t)kt0 * kGemmBK;
    uint32_t phases = 0;  // bit s: parity of stage s's next completion
    bool ok = true;

    // prologue: tiles 0 .. S-2 in flight, one commit group each (empty past KT)
#pragma unroll
    for (int s = 0; s < S - 1; ++s) {
        if (s < KT) {
            load_tile<kGemmBM>(smem_u32(Sm.a[s]), Ab + (size_t)s * kGemmBK, g.lda, rows_a);
            load_tile<BN>(smem_u32(Sm.b[s]), Bb + (size_t)s * kGemmBK, g.ldb, rows_b);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kt = 0; kt < KT; ++kt) {
        const int s = kt % S;
        const int nk = kt + S - 1;
        if (nk < KT) {
            const int sn = nk % S;  // = (kt - 1) % S: the stage tile kt-1's MMAs read
            if (kt >= 1) {
                ok = ok && mbar_wait(smem_u32(&Sm.bar[sn]), (phases >> sn) & 1u);
                phases ^= 1u << sn;
            }
            load_tile<kGemmBM>(smem_u32(Sm.a[sn]), Ab + (size_t)nk * kGemmBK, g.lda, rows_a);
            load_tile<BN>(smem_u32(Sm.b[sn]), Bb + (size_t)nk * kGemmBK, g.ldb, rows_b);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        // S + kt groups committed; all but the newest S-1 done: tile kt's group is
        asm volatile("cp.async.wait_group %0;" ::"n"(S - 1) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // cp.async data -> tensor core reads
        __syncthreads();
        if (threadIdx.x == 0 && ok) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(Sm.a[s]), sb = smem_u32(Sm.b[s]);
#pragma unroll
            for (int k = 0; k < kGemmBK / 16; ++k) {  // K = 16 per MMA: two core matrices along K
                const uint64_t da = umma_desc(sa + k * 256), db = umma_desc(sb + k * 256);
                const uint32_t acc = (kt > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(umma_idesc<BN>()), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&Sm.bar[s]))
                         : "memory");
        }
    }
    // the last commit covers every MMA this thread issued: tile KT-1 is use
    // (KT-1)/S of its stage, whose earlier uses were all waited on above
    if (KT > 0) {
        const int s = (KT - 1) % S;
        ok = ok && mbar_wait(smem_u32(&Sm.bar[s]), (uint32_t)((KT - 1) / S) & 1u);
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok);  // also: every thread is done with the ring before it stages the epilogue

    if (ok) {
        gemm_epilogue<BN, EPI, kGemmThreads / 32>(g, tmem, reinterpret_cast<float*>(Sm.a[0]), m0, n0);
    } else if (threadIdx.x == 0) {
        atomicExch(g.err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

// ---------------------------------------------------------------------------
// TMA-fed, warp-specialised form of the same GEMM (the default where the
// driver's tensor-map encoder is available).
//
// Operands arrive by TMA (cp.async.bulk.tensor, this GPU's own memory, no
// multicast) as 64-wide K tiles in the 128-byte-swizzled K-major layout: a
// row's 64 bf16 (128 bytes) is one swizzle atom row, 8 rows make a 1024-byte
// atom (SBO = 1024), and each 16-wide K step of the MMA starts 32 bytes
// further into the atom.  One thread of warp 0 is the producer: per K tile
// it waits until the stage's previous MMAs are done (the stage's `empty`
// barrier, which tcgen05.commit arrives on), then posts the tile's byte
// count on the stage's `full` barrier and issues the two tile loads, which
// complete it.  One thread of warp 1 issues the MMAs: it waits on `full`,
// issues four tcgen05.mma and commits them to `empty`; after the last tile
// it commits to `done`.  No block barrier inside the K loop.  All four
// warps then run the same epilogue as the cp.async kernel.  Rows past M or
// N are zero-filled by TMA; every wait is bounded as above.
template <int BN>
__host__ __device__ constexpr int tma_stages() {
    return BN >= 256 ? 4 : (BN >= 128 ? 6 : 8);
}

template <int BN>
struct TmaSmem {
    static constexpr int kStages = tma_stages<BN>();
    alignas(1024) unsigned char a[kStages][kGemmBM * kGemmBK * 2];
    alignas(1024) unsigned char b[kStages][BN * kGemmBK * 2];
    alignas(8) uint64_t full[kStages];
    alignas(8) uint64_t empty[kStages];
    alignas(8) uint64_t done;
    uint32_t tmem;
};

// Shared-memory matrix descriptor of a 128-byte-swizzled K-major tile
// (start >> 4; LBO 16 bytes, unused for this layout; SBO 1024 bytes;
// version 1 at bit 46; layout type 2 = SWIZZLE_128B at bit 61).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(16 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// 2-D tile load: the box at (x = K element, y = row) of the tensor map into
// shared memory at dst, completing `bytes` on barrier bar.  x is a multiple
// of 64 elements (128 bytes).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kTmaThreads) k_gemm_bf16_tma(const __grid_constant__ CUtensorMap tma_a,
                                                               const __grid_constant__ CUtensorMap tma_b, GemmArgs g) {
    static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256, "BN: a multiple of 16 in [32, 256]");
    constexpr int S = tma_stages<BN>();
    constexpr uint32_t kTileBytes = (uint32_t)(kGemmBM + BN) * kGemmBK * 2;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TmaSmem<BN>& Sm = *reinterpret_cast<TmaSmem<BN>*>((void*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * BN;
    constexpr uint32_t kCols = BN;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&Sm.tmem)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 32) {
        for (int s = 0; s < S; ++s) {
            mbar_init(smem_u32(&Sm.full[s]), 1);
            mbar_init(smem_u32(&Sm.empty[s]), 1);
        }
        mbar_init(smem_u32(&Sm.done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tma_a) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tma_b) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = Sm.tmem;

    const int kt0 = blockIdx.z * g.kt_split;
    const int KT = min(g.kt_split, g.K / kGemmBK - kt0);
    bool ok = true;
    if (warp == 0 && lane == 0) {  // producer
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % S;
            if (kt >= S) ok = ok && mbar_wait(smem_u32(&Sm.empty[s]), (uint32_t)(kt / S - 1) & 1u);
            const uint32_t full = smem_u32(&Sm.full[s]);
            mbar_arrive_expect_tx(full, kTileBytes);
            tma_load_2d(smem_u32(Sm.a[s]), &tma_a, (kt0 + kt) * kGemmBK, m0, full);
            tma_load_2d(smem_u32(Sm.b[s]), &tma_b, (kt0 + kt) * kGemmBK, n0, full);
        }
    } else if (warp == 1 && lane == 0) {  // MMA issuer
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % S;
            ok = ok && mbar_wait(smem_u32(&Sm.full[s]), (uint32_t)(kt / S) & 1u);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (ok) {
                const uint32_t sa = smem_u32(Sm.a[s]), sb = smem_u32(Sm.b[s]);
#pragma unroll
                for (int k = 0; k < kGemmBK / 16; ++k) {  // 16 bf16 = 32 bytes further into the swizzle atom
                    const uint64_t da = umma_desc_sw128(sa + k * 32), db = umma_desc_sw128(sb + k * 32);
                    const uint32_t acc = (kt > 0 || k > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
                        "l"(da), "l"(db), "r"(umma_idesc<BN>()), "r"(acc)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&Sm.empty[s]))
                         : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&Sm.done))
                     : "memory");
    }
    __syncwarp();
    ok = ok && mbar_wait(smem_u32(&Sm.done), 0u);  // every MMA (and so every load) is done
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok);
    if (ok) {
        static_assert(sizeof(Sm.a) >= (size_t)kTmaThreads * kStageStride * 4, "staging fits in the A stages");
        gemm_epilogue<BN, EPI, kTmaThreads / 32>(g, tmem, reinterpret_cast<float*>(Sm.a[0]), m0, n0);
    } else if (threadIdx.x == 0) {
        atomicExch(g.err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

// Persistent form of the TMA kernel, for GEMMs of more than one wave of
// tiles: one CTA per SM walks its share of the work units (tile, K slice)
// with the accumulator double-buffered in tensor memory (2 x BN columns), so
// the epilogue of unit t runs while the MMAs of unit t + 1 issue.  Warp 0
// (one thread) streams K tiles through the S-stage ring across units; warp 1
// (one thread) issues the MMAs into buffer t & 1, after waiting on that
// buffer's `tempty` barrier (its previous contents read out), and commits the
// unit's last MMAs to `tfull`; warps 2..9 wait on `tfull`, run the epilogue
// out of tensor memory through their own staging area (the ring stays in
// use), and arrive on `tempty` (8 arrivals).  Units run in groups of
// kPersistGroupM row tiles, column tiles within a group, so the CTAs working
// at the same time share operand tiles in L2.  Every wait is bounded; a role
// whose wait gives up records the error and stops, and the others' waits
// then run out in turn.
constexpr int kPersistThreads = 10 * 32;
constexpr int kPersistEpiWarps = 8;  // overlapped with the MMAs, so fewer warps suffice; the ring keeps 4-8 stages
constexpr int kPersistGroupM = 16;

template <int BN>
__host__ __device__ constexpr int persist_stages() {
    return BN >= 256 ? 4 : (BN >= 128 ? 6 : 8);
}

template <int BN>
struct PersistSmem {
    static constexpr int kStages = persist_stages<BN>();
    alignas(1024) unsigned char a[kStages][kGemmBM * kGemmBK * 2];
    alignas(1024) unsigned char b[kStages][BN * kGemmBK * 2];
    alignas(16) float stage[kPersistEpiWarps * 32 * kStageStride];
    alignas(8) uint64_t full[kStages];
    alignas(8) uint64_t empty[kStages];
    alignas(8) uint64_t tfull[2];
    alignas(8) uint64_t tempty[2];
    uint32_t tmem;
};

// Work unit u: K slice z = u / tiles, tile u % tiles in grouped order.
__device__ __forceinline__ void persist_unit(int u, int n_mt, int n_nt, int& mt, int& nt, int& z) {
    const int tiles = n_mt * n_nt;
    z = u / tiles;
    const int t = u - z * tiles;
    const int per_group = kPersistGroupM * n_nt;
    const int grp = t / per_group, r = t - grp * per_group;
    const int gm = min(kPersistGroupM, n_mt - grp * kPersistGroupM);  // rows in this (last) group
    mt = grp * kPersistGroupM + r % gm;
    nt = r / gm;
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kPersistThreads, 1)
    k_gemm_bf16_tma_persistent(const __grid_constant__ CUtensorMap tma_a, const __grid_constant__ CUtensorMap tma_b,
                               GemmArgs g, int n_units, int n_mt, int n_nt) {
    static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256, "BN: a multiple of 16 in [32, 256]");
    constexpr int S = persist_stages<BN>();
    constexpr uint32_t kTileBytes = (uint32_t)(kGemmBM + BN) * kGemmBK * 2;
    constexpr uint32_t kCols = 2 * BN;  // two accumulators
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    PersistSmem<BN>& Sm =
        *reinterpret_cast<PersistSmem<BN>*>((void*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT_all = g.K / kGemmBK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&Sm.tmem)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 32) {
        for (int s = 0; s < S; ++s) {
            mbar_init(smem_u32(&Sm.full[s]), 1);
            mbar_init(smem_u32(&Sm.empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&Sm.tfull[b]), 1);
            mbar_init(smem_u32(&Sm.tempty[b]), kPersistEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tma_a) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tma_b) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = Sm.tmem;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {  // producer: K tiles of every unit through the ring
            uint32_t it = 0;
            for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x) {
                int mt, nt, z;
                persist_unit(u, n_mt, n_nt, mt, nt, z);
                const int kt0 = z * g.kt_split, KT = min(g.kt_split, KT_all - kt0);
                for (int kt = 0; kt < KT && ok; ++kt, ++it) {
                    const uint32_t s = it % S, n = it / S;
                    if (n >= 1) ok = mbar_wait(smem_u32(&Sm.empty[s]), (n - 1) & 1u);
                    if (!ok) break;
                    const uint32_t full = smem_u32(&Sm.full[s]);
                    mbar_arrive_expect_tx(full, kTileBytes);
                    tma_load_2d(smem_u32(Sm.a[s]), &tma_a, (kt0 + kt) * kGemmBK, mt * kGemmBM, full);
                    tma_load_2d(smem_u32(Sm.b[s]), &tma_b, (kt0 + kt) * kGemmBK, nt * BN, full);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            uint32_t it = 0, t = 0;
            for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x, ++t) {
                int mt, nt, z;
                persist_unit(u, n_mt, n_nt, mt, nt, z);
                const int kt0 = z * g.kt_split, KT = min(g.kt_split, KT_all - kt0);
                const uint32_t b = t & 1u, j = t >> 1;  // buffer, its use count
                if (j >= 1) ok = mbar_wait(smem_u32(&Sm.tempty[b]), (j - 1) & 1u);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc_addr = tmem + b * (uint32_t)BN;
                for (int kt = 0; kt < KT; ++kt, ++it) {
                    const uint32_t s = it % S, n = it / S;
                    ok = mbar_wait(smem_u32(&Sm.full[s]), n & 1u);
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = smem_u32(Sm.a[s]), sb = smem_u32(Sm.b[s]);
#pragma unroll
                    for (int k = 0; k < kGemmBK / 16; ++k) {
                        const uint64_t da = umma_desc_sw128(sa + k * 32), db = umma_desc_sw128(sb + k * 32);
                        const uint32_t acc = (kt > 0 || k > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(acc_addr),
                            "l"(da), "l"(db), "r"(umma_idesc<BN>()), "r"(acc)
                            : "memory");
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&Sm.empty[s]))
                                 : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&Sm.tfull[b]))
                             : "memory");
            }
        }
    } else {  // epilogue warps 2 .. 9
        uint32_t t = 0;
        for (int u = blockIdx.x; u < n_units; u += gridDim.x, ++t) {
            int mt, nt, z;
            persist_unit(u, n_mt, n_nt, mt, nt, z);
            const uint32_t b = t & 1u, j = t >> 1;
            ok = mbar_wait(smem_u32(&Sm.tfull[b]), j & 1u);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            gemm_epilogue<BN, EPI, kPersistEpiWarps>(g, tmem + b * (uint32_t)BN, Sm.stage, mt * kGemmBM, nt * BN,
                                                     2);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&Sm.tempty[b]))
                                        : "memory");
        }
    }
    __syncwarp();  // warps 0 and 1 reconverge after their one-thread roles
    if (!ok) atomicExch(g.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

template <int BN>
constexpr size_t gemm_persist_smem_bytes() {
    return sizeof(PersistSmem<BN>) + 1024;
}

template <int BN>
constexpr size_t gemm_tma_smem_bytes() {
    return sizeof(TmaSmem<BN>) + 1024;
}

template <int BN>
constexpr size_t gemm_smem_bytes() {
    return sizeof(GemmSmem<BN>) + 1024;
}

}  // namespace ngpu
