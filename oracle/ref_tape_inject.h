/*
 * ref_tape_inject.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Forced-include header (nvcc -include) used when the oracle recipe compiles
 * the reference's own CUDA sources in place.  After <curand_kernel.h> has been
 * seen, three macros reroute the reference's device RNG calls:
 *
 *   curand_init(seed, subseq, offset, state)  -> remember the particle index
 *   curand_normal(state)                      -> next normal from the tape
 *   curand_normal4(state)                     -> the next four normals
 *   curand_uniform(state)                     -> next uniform from the tape
 *
 * Each particle keeps one normal counter and one uniform counter in the
 * (otherwise unused) ctr fields of its curandStatePhilox4_32_10_t, so the
 * k-th normal drawn by particle i within a tick is tape_normals[k*n + i].  The
 * harness resets the counters before every tick.  A missing tape or a draw
 * past the end of the tape returns a neutral value and raises a flag instead
 * of reading out of bounds.
 */
#ifndef SVPF_REF_TAPE_INJECT_H
#define SVPF_REF_TAPE_INJECT_H

#include <cuda_runtime.h>
#include <curand_kernel.h>

extern __device__ const float* svpf_ref_tape_normals;
extern __device__ const float* svpf_ref_tape_uniforms;
extern __device__ int svpf_ref_tape_n;
extern __device__ int svpf_ref_tape_normal_slots;
extern __device__ int svpf_ref_tape_uniform_slots;
extern __device__ int svpf_ref_tape_flags;   /* bit0: overrun, bit1: no tape */

static __device__ __forceinline__ void svpf_ref_tape_init(unsigned long long seed,
                                                           unsigned long long subsequence,
                                                           unsigned long long offset,
                                                           curandStatePhilox4_32_10_t* st) {
    (void)seed; (void)offset;
    st->ctr.x = (unsigned int)subsequence;  /* particle index */
    st->ctr.y = 0u;                          /* normal draws this tick */
    st->ctr.z = 0u;                          /* uniform draws this tick */
    st->ctr.w = 0u;
}

static __device__ __forceinline__ float svpf_ref_tape_normal(curandStatePhilox4_32_10_t* st) {
    unsigned int k = st->ctr.y++;
    unsigned int i = st->ctr.x;
    const float* tape = svpf_ref_tape_normals;
    if (tape == nullptr) { atomicOr(&svpf_ref_tape_flags, 2); return 0.0f; }
    if (k >= (unsigned int)svpf_ref_tape_normal_slots || i >= (unsigned int)svpf_ref_tape_n) {
        atomicOr(&svpf_ref_tape_flags, 1);
        return 0.0f;
    }
    return tape[(size_t)k * (size_t)svpf_ref_tape_n + i];
}

static __device__ __forceinline__ float svpf_ref_tape_uniform(curandStatePhilox4_32_10_t* st) {
    unsigned int k = st->ctr.z++;
    unsigned int i = st->ctr.x;
    const float* tape = svpf_ref_tape_uniforms;
    if (tape == nullptr) { atomicOr(&svpf_ref_tape_flags, 2); return 1.0f; }
    if (k >= (unsigned int)svpf_ref_tape_uniform_slots || i >= (unsigned int)svpf_ref_tape_n) {
        atomicOr(&svpf_ref_tape_flags, 1);
        return 1.0f;
    }
    return tape[(size_t)k * (size_t)svpf_ref_tape_n + i];
}

/* curand_normal4: four consecutive normal slots (x, y, z, w). */
static __device__ __forceinline__ float4 svpf_ref_tape_normal4(curandStatePhilox4_32_10_t* st) {
    float4 r;
    r.x = svpf_ref_tape_normal(st);
    r.y = svpf_ref_tape_normal(st);
    r.z = svpf_ref_tape_normal(st);
    r.w = svpf_ref_tape_normal(st);
    return r;
}

#define curand_init(a, b, c, d) svpf_ref_tape_init((a), (b), (c), (d))
#define curand_normal4(s) svpf_ref_tape_normal4(s)
#define curand_normal(s) svpf_ref_tape_normal(s)
#define curand_uniform(s) svpf_ref_tape_uniform(s)

#endif
