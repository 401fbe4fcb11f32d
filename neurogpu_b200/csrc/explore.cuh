// Parameter-exploration score of many voltage traces, one thread per trace:
// the number of peaks of dV/dt that scipy.signal.find_peaks(dvdt, height,
// distance) returns (scipy 1.x; not vendored in the reference).  This is the
// score of the reference's exploration run (GUI/plot_param_explor.py:77-107:
// dvdt = numpy.diff(v) / dt, find_peaks(dvdt, 15, distance=5), the count),
// computed where the traces lie instead of on the host after a 554 MB
// VHotP0.dat readback.
//
// The steps are scipy's published ones:
//   1. local maxima of x = dvdt: x[i-1] < x[i] followed by a run of samples
//      equal to x[i] and then a smaller sample; the peak is the middle of the
//      run ((first + last) // 2); first and last samples never peak;
//   2. heights: keep peaks with x >= height;
//   3. distance: visit peaks by decreasing height and remove every peak
//      closer than `distance` samples to a kept one (equal heights: the later
//      peak first, which is the order of a stable sort; scipy leaves the order
//      of ties to numpy's unstable argsort).
// Step 3 is done per cluster (a maximal run of peaks whose neighbours are
// closer than `distance`): peaks of different clusters never remove each
// other.
//
// dvdt is computed as here in double from the float32 trace: ((double)v[j+1]
// - (double)v[j]) / dt, the value numpy computes from the same samples read
// as float64 (the difference of two float32 values in this range is exact
// in double and the quotient is correctly rounded), so every comparison
// matches.
//
// Scratch: the candidate peaks' sample positions, [cap][n_traces] int32 with
// cap = n_samples / 2 + 1 (peaks are at least two samples apart), written and
// read by the trace's own thread only; threads of a warp touch one row at a
// time, consecutive traces.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ngpu {

struct PeakArgs {
    const float* v;
    int64_t stride_trace, stride_sample;
    int n_traces, n_samples;
    double dt, height;
    int distance;
    int32_t* pos;      // scratch [cap][n_traces]
    int cap;
    int32_t* out;      // [n_traces] peak counts
};

__host__ __device__ inline int peak_scratch_cap(int n_samples) { return n_samples / 2 + 1; }

__host__ __device__ __forceinline__ double dvdt_at(const PeakArgs& a, const float* v, int j) {
    return ((double)v[(int64_t)(j + 1) * a.stride_sample] - (double)v[(int64_t)j * a.stride_sample]) / a.dt;
}

// Removed peaks carry kPeakGone in their position word, kept ones kPeakKept.
constexpr int32_t kPeakGone = 1 << 30, kPeakKept = 1 << 29;
// Samples loaded ahead per thread (rows in flight; the scan is latency-bound).
constexpr int kPeakChunk = 32;

// The score of trace t (one thread's work; host-callable for tests).
__host__ __device__ inline int dvdt_peaks_trace(const PeakArgs& a, int t) {
    const float* v = a.v + (int64_t)t * a.stride_trace;
    int32_t* pos = a.pos + t;
    const int64_t ps = a.n_traces;
    const int nx = a.n_samples - 1;  // dvdt samples
    // 1 + 2: local maxima at or above the height, in position order.  One
    // pass over the samples, kPeakChunk loads in flight: x[j] is formed from
    // samples j and j + 1 as they arrive, and a candidate is a rising sample
    // (x[j-1] < x[j], 1 <= j <= nx - 2) whose run of equal values ends in a
    // smaller sample (a peak at the run's middle), in a larger one (no peak;
    // that sample is the next candidate) or in a NaN or the trace's end (no
    // peak).  These are the decisions of scipy's scan, taken as the samples
    // stream by instead of by looking ahead.
    int m = 0;
    if (nx >= 3) {
        float vprev = v[0];
        double xprev = 0.0, pv = 0.0;
        bool cand = false;
        int i0 = 0;
        for (int s0 = 1; s0 < a.n_samples; s0 += kPeakChunk) {
            float buf[kPeakChunk];
#pragma unroll
            for (int u = 0; u < kPeakChunk; ++u)
                if (s0 + u < a.n_samples) buf[u] = v[(int64_t)(s0 + u) * a.stride_sample];
#pragma unroll
            for (int u = 0; u < kPeakChunk; ++u) {
                const int j = s0 + u - 1;  // dvdt sample of samples j, j + 1
                if (j + 1 < a.n_samples) {
                    const double x = ((double)buf[u] - (double)vprev) / a.dt;
                    vprev = buf[u];
                    if (j > 0) {
                        if (cand) {
                            if (x == pv) {
                                // the run goes on
                            } else if (x < pv) {
                                if (pv >= a.height && m < a.cap) pos[(int64_t)m++ * ps] = (i0 + j - 1) / 2;
                                cand = false;
                            } else if (x > pv) {
                                cand = j <= nx - 2;
                                i0 = j;
                                pv = x;
                            } else {
                                cand = false;  // NaN
                            }
                        } else if (xprev < x && j <= nx - 2) {
                            cand = true;
                            i0 = j;
                            pv = x;
                        }
                    }
                    xprev = x;
                }
            }
        }
    }
    // 3: distance, cluster by cluster
    const int d = a.distance;
    int kept = 0;
    int c0 = 0;
    while (c0 < m) {
        int c1 = c0 + 1;
        while (c1 < m && pos[(int64_t)c1 * ps] - pos[(int64_t)(c1 - 1) * ps] < d) ++c1;
        if (c1 - c0 == 1) {
            ++kept;
        } else {
            // greedy by height over the cluster [c0, c1): the open peak of
            // largest (height, position) is kept and its close neighbours go
            for (;;) {
                int best = -1;
                double hb = 0.0;
                for (int k = c0; k < c1; ++k) {
                    const int32_t p = pos[(int64_t)k * ps];
                    if (p & (kPeakGone | kPeakKept)) continue;
                    const double h = dvdt_at(a, v, p);
                    if (best < 0 || h >= hb) {  // equal heights: the later peak
                        best = k;
                        hb = h;
                    }
                }
                if (best < 0) break;
                const int32_t pb = pos[(int64_t)best * ps];
                pos[(int64_t)best * ps] = pb | kPeakKept;
                ++kept;
                for (int k = best - 1; k >= c0; --k) {
                    const int32_t p = pos[(int64_t)k * ps];
                    if (pb - (p & (kPeakKept - 1)) >= d) break;
                    pos[(int64_t)k * ps] = p | kPeakGone;
                }
                for (int k = best + 1; k < c1; ++k) {
                    const int32_t p = pos[(int64_t)k * ps];
                    if ((p & (kPeakKept - 1)) - pb >= d) break;
                    pos[(int64_t)k * ps] = p | kPeakGone;
                }
            }
        }
        c0 = c1;
    }
    return kept;
}

__global__ void __launch_bounds__(64) k_dvdt_peaks(const PeakArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < a.n_traces) a.out[t] = dvdt_peaks_trace(a, t);
}

}  // namespace ngpu
