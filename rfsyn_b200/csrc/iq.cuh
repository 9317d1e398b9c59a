// iq.cuh -- the FDTD stage's output signal and rfsyn's AWGN stage, computed
// on the device from a resident probe series (included by engine.cu).
//
// rfsyn's chain turns the probe series into a complex float signal
// (cli/fdtd_stage.c:23-24: (float)probe[n] + 0i), adds white Gaussian noise
// (engine/noise/awgn.c:16-44) and writes the samples as interleaved float32
// I/Q (cli/main.c:70-85).  Here the signal never leaves the GPU until the
// finished I/Q samples are copied back:
//   k_iq_power -- one thread: the mean power sum_n |x_n|^2 / N in double, in
//     rfsyn's order (a sequential sum, so the noise scale is bit-identical),
//     then per_axis_std = sqrt(P / snr_linear / 2);
//   k_iq_noise -- one thread per sample: rfsyn draws u1, u2 for sample n as
//     the outputs 2n and 2n+1 of one PCG32 stream (engine/core/rng.c); each
//     thread jumps its own copy of the generator ahead by 2n steps (the LCG
//     step composes: x -> a x + c applied d times is x -> A x + C, A and C by
//     repeated squaring; Brown, "Random number generation with arbitrary
//     strides", Trans. Am. Nucl. Soc. 1994), then forms the Box-Muller pair
//     with rfsyn's float operation order.  logf, cosf and sinf of a float are
//     taken as the float rounding of CUDA's double-precision log, cos and sin,
//     which is the correctly rounded float result except in rare ties.
#pragma once

namespace rfb {

constexpr unsigned long long PCG_MULT = 6364136223846793005ULL;

struct Pcg32 {
    unsigned long long state, inc;
};

__host__ __device__ __forceinline__ unsigned pcg32_next(Pcg32 &g) {
    const unsigned long long old = g.state;
    g.state = old * PCG_MULT + g.inc;
    const unsigned xs = (unsigned)(((old >> 18u) ^ old) >> 27u);
    const unsigned rot = (unsigned)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}

// rng_seed (rng.c:3-9)
__host__ __device__ __forceinline__ Pcg32 pcg32_seeded(unsigned long long seed, unsigned long long stream) {
    Pcg32 g{0ULL, (stream << 1u) | 1u};
    pcg32_next(g);
    g.state += seed;
    pcg32_next(g);
    return g;
}

// The generator after `delta` more steps.
__host__ __device__ __forceinline__ void pcg32_advance(Pcg32 &g, unsigned long long delta) {
    unsigned long long acc_mult = 1ULL, acc_plus = 0ULL, cur_mult = PCG_MULT, cur_plus = g.inc;
    while (delta) {
        if (delta & 1ULL) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1ULL) * cur_plus;
        cur_mult *= cur_mult;
        delta >>= 1;
    }
    g.state = acc_mult * g.state + acc_plus;
}

// rng_uniform (rng.c:20-23): 24 random bits / 2^24
__device__ __forceinline__ float pcg32_uniform(Pcg32 &g) { return (float)(pcg32_next(g) >> 8) / (float)(1u << 24); }

template <typename T>
__global__ void k_iq_power(const T *x, long long n, double snr_linear, double *std_out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double p = 0.0;
    for (long long q = 0; q < n; q++) {
        const float mag = fabsf((float)x[q]);
        p = __dadd_rn(p, __dmul_rn((double)mag, (double)mag));
    }
    p = p / (double)n;
    const double noise = snr_linear > 0.0 ? p / snr_linear : 0.0;
    *std_out = sqrt(noise / 2.0);
}

// out[2n], out[2n+1]: I and Q of sample n; noise only when std_in != nullptr.
template <typename T>
__global__ void k_iq_noise(const T *x, long long n, const double *std_in, unsigned long long seed,
                           unsigned long long stream, float *out) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float xi = (float)x[q];
    if (!std_in) {
        out[2 * q] = xi;
        out[2 * q + 1] = 0.0f;
        return;
    }
    Pcg32 g = pcg32_seeded(seed, stream);
    pcg32_advance(g, 2ULL * (unsigned long long)q);
    float u1 = pcg32_uniform(g);
    const float u2 = pcg32_uniform(g);
    if (u1 <= 0.0f) u1 = 1e-9f;
    const float r = __fsqrt_rn(__fmul_rn(-2.0f, (float)log((double)u1)));
    const float t = __fmul_rn(__fmul_rn(2.0f, (float)3.14159265358979323846), u2);
    const float sd = (float)*std_in;
    const float nre = __fmul_rn(__fmul_rn(sd, r), (float)cos((double)t));
    const float nim = __fmul_rn(__fmul_rn(sd, r), (float)sin((double)t));
    out[2 * q] = __fadd_rn(xi, nre);
    out[2 * q + 1] = __fadd_rn(0.0f, nim);
}

}  // namespace rfb
