// Spike / ISI / amplitude / AHP / voltage features of many voltage traces,
// one thread per trace.
//
// The reference extracts features trace by trace on a CPU pool (eFEL through
// P/efel_ext.py:23-96, GUI/score_functions.py); here a trace never leaves the
// GPU: the kernel reads the simulator's trace buffer where it lies.  Traces
// are addressed with two strides, element (trace t, sample s) at
// v[t * stride_trace + s * stride_sample]: the simulator's buffer is
// sample-major ([sample][site][instance], stride_trace 1), so at each sample
// the threads of a warp read 32 consecutive instances, one coalesced row, and
// every thread walks its own trace forward in time.  Pass 1 finds the upward
// threshold crossings inside the stimulus window and accumulates ISIs, the
// maximum and minimum of each inter-crossing segment (AP peaks, AHP troughs)
// and the window statistics; pass 2 counts the samples at or above the
// half-amplitude level, which needs pass 1's mean peak and trough.
//
// The definitions are those of neurogpu_b200/features.py (the batched torch
// statement the surrogate network is trained on), feature for feature:
// crossing times (index + 1) * dt in float32 as there, sums in FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ngpu {

constexpr int kNFeatures = 20;

struct FeatureArgs {
    const float* v;
    int64_t stride_trace, stride_sample;
    int n_traces, n_samples;
    float dt, threshold;
    float dur;               // (i_off - i_on) dt
    int i_on, i_off;         // stimulus window [i_on, i_off) in samples
    int vb_lo, vb_hi;        // voltage_base window
    int ss_lo, ss_hi;        // steady-state window
    int af_lo, af_hi;        // after-stimulus window (af_lo < 0: the last sample)
    float* out;              // [n_traces][20]
};

// Samples are read kChunk at a time into registers, all loads of a chunk
// issued before any is used: kChunk rows in flight per thread.
constexpr int kChunk = 16;

template <typename F>
__device__ __forceinline__ void for_samples(const float* v, int64_t st, int lo, int hi, F&& f) {
    for (int j0 = lo; j0 < hi; j0 += kChunk) {
        float x[kChunk];
#pragma unroll
        for (int u = 0; u < kChunk; ++u)
            if (j0 + u < hi) x[u] = v[(int64_t)(j0 + u) * st];
#pragma unroll
        for (int u = 0; u < kChunk; ++u)
            if (j0 + u < hi) f(j0 + u, x[u]);
    }
}

__device__ __forceinline__ double win_mean(const float* v, int64_t st, int lo, int hi) {
    double s = 0;
    for_samples(v, st, lo, hi, [&](int, float x) { s += (double)x; });
    return hi > lo ? s / (double)(hi - lo) : 0.0;
}

__global__ void __launch_bounds__(128) k_trace_features(const FeatureArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n_traces) return;
    const float* v = a.v + (int64_t)t * a.stride_trace;
    const int64_t st = a.stride_sample;
    const float TH = a.threshold, dt = a.dt;
    const int W = a.i_off - a.i_on;
    const float dur = a.dur;
    // pass 1
    float vmax = -INFINITY;
    for_samples(v, st, 0, a.i_on, [&](int, float x) { vmax = fmaxf(vmax, x); });
    for_samples(v, st, a.i_off, a.n_samples, [&](int, float x) { vmax = fmaxf(vmax, x); });
    float wmin = INFINITY, wmax = -INFINITY;
    double wsum = 0, wsq = 0;
    int n = 0, first_idx = -1;
    float first_t = 0, last_t = 0, first_isi = 0, last_isi = 0;
    double isi_sum = 0, isi_sq = 0;
    float seg_max = -INFINITY, seg_min = INFINITY;
    double pk_sum = 0, pk_sq = 0, tr_sum = 0;
    float prev = 0;
    for_samples(v + (int64_t)a.i_on * st, st, 0, W, [&](int j, float x) {
        vmax = fmaxf(vmax, x);
        wmin = fminf(wmin, x);
        wmax = fmaxf(wmax, x);
        wsum += x;
        wsq += (double)x * x;
        if (j > 0 && prev < TH && x >= TH) {  // crossing between samples j-1 and j: t = j dt
            const float tc = (float)j * dt;
            if (n > 0) {                      // the previous segment ends
                pk_sum += seg_max;
                pk_sq += (double)seg_max * seg_max;
                tr_sum += seg_min;
                const float isi = tc - last_t;
                isi_sum += isi;
                isi_sq += (double)isi * isi;
                if (n == 1) first_isi = isi;
                last_isi = isi;
            } else {
                first_t = tc;
                first_idx = j;
            }
            last_t = tc;
            ++n;
            seg_max = -INFINITY;
            seg_min = INFINITY;
        }
        if (n > 0) {
            seg_max = fmaxf(seg_max, x);
            seg_min = fminf(seg_min, x);
        }
        prev = x;
    });
    if (n > 0) {
        pk_sum += seg_max;
        pk_sq += (double)seg_max * seg_max;
        tr_sum += seg_min;
    }
    const bool has1 = n >= 1, has2 = n >= 2;
    const double nd = (double)n;
    const double n_isi = (double)(n - 1);
    const double mean_isi = has2 ? isi_sum / n_isi : (double)dur;
    double isi_cv = 0;
    if (has2) {
        const double var = fmax(0.0, isi_sq / n_isi - mean_isi * mean_isi);
        isi_cv = sqrt(var) / fmax(mean_isi, 1e-6);
    }
    const double pk_mean = has1 ? pk_sum / nd : (double)wmax;
    const double pk_std = has1 ? sqrt(fmax(0.0, pk_sq / nd - pk_mean * pk_mean)) : 0.0;
    const double ahp = has1 ? tr_sum / nd : (double)wmin;
    const float half = (float)(0.5 * (pk_mean + ahp));
    // pass 2: samples at or above half amplitude after the first crossing
    int above = 0;
    if (has1) for_samples(v + (int64_t)a.i_on * st, st, first_idx, W, [&](int, float x) { above += x >= half ? 1 : 0; });
    const double wmean = W > 0 ? wsum / W : 0.0;
    const double wstd = W > 1 ? sqrt(fmax(0.0, (wsq - (double)W * wmean * wmean) / (double)(W - 1))) : 0.0;
    float* o = a.out + (int64_t)t * kNFeatures;
    o[0] = (float)n;
    o[1] = has1 ? first_t : dur;
    o[2] = (float)mean_isi;
    o[3] = (float)isi_cv;
    o[4] = has2 ? first_isi : dur;
    o[5] = has2 ? last_isi : dur;
    o[6] = has2 ? last_isi / fmaxf(first_isi, 1e-6f) : 1.0f;
    o[7] = (float)pk_mean;
    o[8] = (float)pk_std;
    o[9] = (float)ahp;
    o[10] = (float)(pk_mean - ahp);
    o[11] = has1 ? (float)above * dt / (float)n : 0.0f;
    o[12] = (float)win_mean(v, st, a.vb_lo, a.vb_hi);
    o[13] = (float)win_mean(v, st, a.ss_lo, a.ss_hi);
    o[14] = a.af_lo < 0 ? v[(int64_t)(a.n_samples - 1) * st] : (float)win_mean(v, st, a.af_lo, a.af_hi);
    o[15] = vmax;
    o[16] = wmin;
    o[17] = (float)wmean;
    o[18] = (float)wstd;
    o[19] = has1 ? last_t : dur;
}

}  // namespace ngpu
