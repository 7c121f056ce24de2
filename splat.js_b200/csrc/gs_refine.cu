// gs_refine.cu -- MCMC-lite relocation and growth (trainer.js:666-794) on the
// device.
//
// The reference reads the whole model back to the CPU, edits it in
// JavaScript and writes it all back (six full-buffer round trips).  Here:
//   1. k_refine_classify: dead (sigmoid(opacity) < 0.02) / donor (> 0.4)
//      flags and each donor's descending mean-log-scale sort key, computed
//      in double as the JavaScript does;
//   2. stable compaction (scan) of the dead and donor index lists, and a
//      stable radix sort of the donors by mean log-scale, descending -- the
//      reference's [...donors].sort(...) (Array.prototype.sort is stable);
//   3. the host reads three counts, draws rng() in the reference's order and
//      uploads a plan (donor list position, split flag, three Gaussian
//      jitters per spawn); with opacity-weighted donor sampling it also reads
//      the donors' opacity logits (k_donor_opacity) to build the weights;
//   4. k_refine_apply writes every spawned splat in parallel.  A donor that
//      was split by an earlier spawn of the same call is read as the
//      reference would see it then (log-scales shrunk by log(1/1.6)): each
//      donor's split sequence number is scattered first, so the sequential
//      dependence of the reference's loop is resolved without a sequential
//      pass;
//   5. k_refine_split_donors applies the split donors' own shrink and clears
//      their moments.
// Float32Array stores in the reference round each double result to f32;
// the (float) casts below do the same.
#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {

__device__ __forceinline__ uint64_t desc_key(double d) {
  uint64_t u = (uint64_t)__double_as_longlong(d);
  const uint64_t asc = (u >> 63) ? ~u : (u | 0x8000000000000000ull);
  return ~asc;
}

__global__ void k_refine_classify(const float* params, uint32_t n, uint32_t* deadFlag, uint32_t* donorFlag) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = (double)params[(size_t)i * 16 + 13];
  const double o = 1.0 / (1.0 + exp(-x));
  const bool dead = o < 0.02;
  deadFlag[i] = dead ? 1u : 0u;
  donorFlag[i] = (!dead && o > 0.4) ? 1u : 0u;
}

__global__ void k_refine_compact(const float* params, uint32_t n, const uint32_t* deadFlag,
                                 const uint32_t* deadOff, const uint32_t* donorFlag, const uint32_t* donorOff,
                                 uint32_t* deadList, uint32_t* donorList, uint64_t* donorKeys,
                                 uint32_t* donorVals) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (deadFlag[i]) deadList[deadOff[i]] = i;
  if (donorFlag[i]) {
    const uint32_t o = donorOff[i];
    donorList[o] = i;
    const float* p = params + (size_t)i * 16;
    const double mls = ((double)p[3] + (double)p[4] + (double)p[5]) / 3.0;
    donorKeys[o] = desc_key(mls);
    donorVals[o] = i;
  }
}

__global__ void k_refine_split_seq(const RefineSpawn* plan, uint32_t count, const uint32_t* bigSorted,
                                   uint32_t* splitSeq) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  if (plan[s].split) splitSeq[bigSorted[plan[s].pos]] = s;
}

__global__ void k_refine_apply(RefineApplyArgs a) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.count) return;
  const RefineSpawn sp = a.plan[s];
  const uint32_t target = s < a.moved ? a.deadList[s] : a.n + (s - a.moved);
  const uint32_t don = sp.split ? a.bigSorted[sp.pos] : a.donorList[sp.pos];
  const float* pd = a.params + (size_t)don * 16;
  float* pt = a.params + (size_t)target * 16;
  const double shrink = log(1.0 / 1.6);
  // the donor as the reference's loop sees it at this spawn
  float ls[3] = {pd[3], pd[4], pd[5]};
  if (a.splitSeq[don] < s)
    for (int k = 0; k < 3; ++k) ls[k] = (float)((double)ls[k] + shrink);
  const double sc = exp(((double)ls[0] + (double)ls[1] + (double)ls[2]) / 3.0);
  float out[16];
  for (int k = 0; k < 3; ++k) out[k] = (float)((double)pd[k] + sp.g[k] * sc * 0.7);
  for (int k = 0; k < 3; ++k) out[3 + k] = ls[k];
  for (int k = 6; k <= 12; ++k) out[k] = pd[k];
  if (sp.split) {
    for (int k = 3; k <= 5; ++k) out[k] = (float)((double)out[k] + shrink);
    out[13] = pd[13];
  } else {
    for (int k = 3; k <= 5; ++k) out[k] = (float)((double)out[k] + log(0.85));
    out[13] = (float)log(0.25 / 0.75);
  }
  out[14] = 0.0f;
  out[15] = 0.0f;
  for (int k = 0; k < 16; ++k) {
    pt[k] = out[k];
    a.m[(size_t)target * 16 + k] = 0.0f;
    a.v[(size_t)target * 16 + k] = 0.0f;
  }
  const int shr = a.shr;
  for (int k = 0; k < shr; ++k) {
    a.sh[(size_t)target * shr + k] = a.sh[(size_t)don * shr + k];
    a.shM[(size_t)target * shr + k] = 0.0f;
    a.shV[(size_t)target * shr + k] = 0.0f;
  }
}

__global__ void k_refine_split_donors(RefineApplyArgs a) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.count) return;
  const RefineSpawn sp = a.plan[s];
  if (!sp.split) return;
  const uint32_t don = a.bigSorted[sp.pos];
  float* pd = a.params + (size_t)don * 16;
  const double shrink = log(1.0 / 1.6);
  for (int k = 3; k <= 5; ++k) pd[k] = (float)((double)pd[k] + shrink);
  for (int k = 0; k < 16; ++k) {
    a.m[(size_t)don * 16 + k] = 0.0f;
    a.v[(size_t)don * 16 + k] = 0.0f;
  }
  for (int k = 0; k < a.shr; ++k) {
    a.shM[(size_t)don * a.shr + k] = 0.0f;
    a.shV[(size_t)don * a.shr + k] = 0.0f;
  }
}

// opacity logits of the compacted donors, in donor-list order (the weights
// of opacity-weighted donor sampling)
__global__ void k_donor_opacity(const float* params, const uint32_t* donorList, uint32_t nDonors, float* out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nDonors) out[k] = params[(size_t)donorList[k] * 16 + 13];
}

__global__ void k_max_u32(const uint32_t* x, uint32_t count, uint32_t* out) {
  uint32_t m = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) m = max(m, x[i]);
  m = __reduce_max_sync(0xFFFFFFFFu, m);
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

void launch_refine_classify(const float* params, uint32_t n, uint32_t* deadFlag, uint32_t* donorFlag,
                            cudaStream_t s) {
  if (n) k_refine_classify<<<(n + 255) / 256, 256, 0, s>>>(params, n, deadFlag, donorFlag);
}
void launch_refine_compact(const float* params, uint32_t n, const uint32_t* deadFlag, const uint32_t* deadOff,
                           const uint32_t* donorFlag, const uint32_t* donorOff, uint32_t* deadList,
                           uint32_t* donorList, uint64_t* donorKeys, uint32_t* donorVals, cudaStream_t s) {
  if (n)
    k_refine_compact<<<(n + 255) / 256, 256, 0, s>>>(params, n, deadFlag, deadOff, donorFlag, donorOff, deadList,
                                                     donorList, donorKeys, donorVals);
}
void launch_refine_apply(const RefineApplyArgs& a, uint32_t* splitSeq, cudaStream_t s) {
  if (!a.count) return;
  const unsigned g = (a.count + 255) / 256;
  k_refine_split_seq<<<g, 256, 0, s>>>(a.plan, a.count, a.bigSorted, splitSeq);
  k_refine_apply<<<g, 256, 0, s>>>(a);
  k_refine_split_donors<<<g, 256, 0, s>>>(a);
}
void launch_donor_opacity(const float* params, const uint32_t* donorList, uint32_t nDonors, float* out,
                          cudaStream_t s) {
  if (nDonors) k_donor_opacity<<<(nDonors + 255) / 256, 256, 0, s>>>(params, donorList, nDonors, out);
}
void launch_max_u32(const uint32_t* x, uint32_t count, uint32_t* out, cudaStream_t s) {
  cudaMemsetAsync(out, 0, 4, s);
  if (count) k_max_u32<<<64, 256, 0, s>>>(x, count, out);
}

}  // namespace gs
