// SPDX-License-Identifier: Apache-2.0
// Between-step calls of the drop-in, outside the step graph: the port (ports.py: absorb, emit, retire), the
// liquid's kinetic + gravity energy per world (runtime.py:66-79, 423-430) and the per-world stable step
// (runtime.py:55-62, 82-90, 411-421). All take the caller's particle order.
//
// Port layout: the reference keeps each world's held particles on a stack of [W][max world size]; here the stack of
// world w lives in that world's own index range [ws[w], ws[w + 1]) of one [n] array (a world never holds more
// particles than it has), so the port costs 4 bytes per particle whatever the spread of world sizes.
#pragma once

#include "dfsph_kernels.cuh"
#include "dfsph_reduce.cuh"

namespace adf {

constexpr int8_t PH_LIQUID = 1, PH_RETIRED = -2, PH_HELD = -3;  // config.py:31-35

// Exclusive prefix sum over a 256-thread block (thread order); `total` receives the block's sum.
__device__ __forceinline__ int block_excl_scan256(int v, int* sm, int& total) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(full, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[wid] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int g = 0; g < 8; ++g) {
      const int c = sm[g];
      sm[g] = acc;
      acc += c;
    }
    sm[8] = acc;
  }
  __syncthreads();
  const int r = sm[wid] + x - v;
  total = sm[8];
  __syncthreads();
  return r;
}

// Sum of an int64 over a 256-thread block (exact integers: the order does not matter); valid in thread 0.
__device__ __forceinline__ long long block_sum256_ll(long long v, long long* sm) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  long long s = 0;
  if (threadIdx.x == 0)
    for (int g = 0; g < 8; ++g) s += sm[g];
  return s;
}

// ports.py:_take_kernel, one 256-thread block per world: the world's particles in index order, 256 at a time, an
// ordered block scan giving each taken particle its stack slot, so the stack order equals the reference's serial
// walk. The masked liquid leaves: ACTIVE cleared, velocity zeroed, mass (int64 fixed point, exact) to the world's
// mass_out; with `keep` it is held on the world's stack (absorb), else retired for good (retire).
__global__ void __launch_bounds__(256) k_port_take(const int* __restrict__ ws, const int32_t* __restrict__ mask,
                                                   int keep, int32_t* flags, int8_t* phase,
                                                   const float* __restrict__ mass, float* qd, int* stack, int* top,
                                                   int* taken, int* total, long long* mass_out) {
  __shared__ int sm[9];
  __shared__ long long sml[8];
  const int w = blockIdx.x;
  const int b = ws[w], e = ws[w + 1];
  int t = top[w], k = 0;
  long long out = 0;
  for (int base = b; base < e; base += 256) {
    const int i = base + threadIdx.x;
    const bool take = i < e && mask[i] != 0 && (flags[i] & FLAG_ACTIVE) != 0 && phase[i] >= 1;
    int cnt;
    const int off = block_excl_scan256(take ? 1 : 0, sm, cnt);
    if (take) {
      flags[i] &= ~FLAG_ACTIVE;
      qd[3 * (size_t)i] = 0.0f;
      qd[3 * (size_t)i + 1] = 0.0f;
      qd[3 * (size_t)i + 2] = 0.0f;
      out += to_fixed(mass[i]);
      if (keep) {
        phase[i] = PH_HELD;
        stack[b + t + off] = i;  // < e: a held particle is not liquid, so each particle is on the stack at most once
      } else {
        phase[i] = PH_RETIRED;
      }
    }
    if (keep) t += cnt;
    k += cnt;
  }
  const long long s = block_sum256_ll(out, sml);
  if (threadIdx.x == 0) {
    mass_out[w] += s;
    top[w] = t;
    taken[w] = k;
    total[w] += k;
  }
}

// ports.py:_emit_kernel, one block per world: request r (r < min(n_req[w], R, held)) pops the stack's (r + 1)-th
// particle from the top, as the reference's serial loop does, which becomes liquid at pos[w][r] with vel[w][r]
// (world frame, written into the caller's state).
__global__ void __launch_bounds__(256) k_port_emit(const int* __restrict__ ws, const float* __restrict__ pos,
                                                   const float* __restrict__ vel, int R,
                                                   const int32_t* __restrict__ n_req, float* q, float* qd,
                                                   int32_t* flags, int8_t* phase, const float* __restrict__ mass,
                                                   const int* __restrict__ stack, int* top, int* granted, int* total,
                                                   long long* mass_in) {
  __shared__ long long sml[8];
  const int w = blockIdx.x;
  const int b = ws[w], t0 = top[w];
  const int req = max(min(min(n_req[w], R), t0), 0);
  long long in = 0;
  for (int r = threadIdx.x; r < req; r += blockDim.x) {
    const int i = stack[b + t0 - 1 - r];
    const size_t src = ((size_t)w * R + r) * 3, dst = 3 * (size_t)i;
    q[dst] = pos[src];
    q[dst + 1] = pos[src + 1];
    q[dst + 2] = pos[src + 2];
    qd[dst] = vel[src];
    qd[dst + 1] = vel[src + 1];
    qd[dst + 2] = vel[src + 2];
    flags[i] |= FLAG_ACTIVE;
    phase[i] = PH_LIQUID;
    in += to_fixed(mass[i]);
  }
  const long long s = block_sum256_ll(in, sml);
  if (threadIdx.x == 0) {
    mass_in[w] += s;
    top[w] = t0 - req;
    granted[w] = req;
    total[w] += req;
  }
}

// ports.py:205-216: the masked worlds' reservoir back to its build-time particles, counters to zero.
__global__ void __launch_bounds__(256) k_port_reset(int W, const int* __restrict__ ws, const uint8_t* __restrict__ mask,
                             const int* __restrict__ stack0, const int* __restrict__ top0, int* stack, int* top,
                             int* absorbed, int* emitted, int* retired, int* taken, int* granted) {
  const int w = blockIdx.x;
  if (w >= W || !mask[w]) return;
  for (int i = ws[w] + threadIdx.x; i < ws[w + 1]; i += blockDim.x) stack[i] = stack0[i];
  if (threadIdx.x == 0) {
    top[w] = top0[w];
    absorbed[w] = emitted[w] = retired[w] = taken[w] = granted[w] = 0;
  }
}

// runtime.py:66-79 (_energy_kernel) summed per world as energy_per_world (runtime.py:423-430): one block per
// 256-particle chunk of the reductions' chunk table; e_i = m (v.v / 2 - g.(x - z_ref e_z)) in float64 from the
// float32 dot products the reference forms, folded in the fixed tree of the other per-world sums; the world step is
// k_world_check's.
__global__ void __launch_bounds__(256) k_energy_chunk(DevP P, const float* __restrict__ q,
                                                      const float* __restrict__ qd, const double* __restrict__ z_ref) {
  __shared__ double smd[8];
  const int c = blockIdx.x;
  const int i = P.chunk_begin[c] + threadIdx.x;
  double e = 0.0;
  if (i < P.chunk_end[c] && is_fluid_orig(P, i)) {
    const int w = P.world[i];
    const float* g = P.gravity + 3 * (size_t)w;
    const size_t b = 3 * (size_t)i;
    const float vx = qd[b], vy = qd[b + 1], vz = qd[b + 2];
    const float dz = (float)((double)q[b + 2] - z_ref[w]);
    const float vv = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
    const float gd = __fadd_rn(__fadd_rn(__fmul_rn(g[0], q[b]), __fmul_rn(g[1], q[b + 1])), __fmul_rn(g[2], dz));
    e = (double)P.mass[i] * (0.5 * (double)vv - (double)gd);
  }
  const double s = fold256(e, smd);
  if (threadIdx.x == 0) {
    P.part_sum[c] = s;
    P.part_max[c] = 0.0f;
  }
}

// runtime.py:82-90 (_speed_only_kernel): per-world max |v| of the liquid, non-finite speeds as 1e30; float bits of
// non-negative values order as integers, so an integer atomicMax is the float max.
__global__ void k_speed_max(DevP P, const float* __restrict__ qd, int* speed_bits) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n || !is_fluid_orig(P, i)) return;
  const size_t b = 3 * (size_t)i;
  const float vx = qd[b], vy = qd[b + 1], vz = qd[b + 2];
  float s = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz)));
  if (!isfinite(s)) s = 1.0e30f;
  atomicMax(&speed_bits[P.world[i]], __float_as_int(s));
}

// runtime.py:55-62 (_stable_dt_kernel): dt_max at rest, else clamp(cfl spacing / v, dt_min, dt_max).
__global__ void k_stable_dt(int W, const int* __restrict__ speed_bits, float cfl, float spacing, float dt_min,
                            float dt_max, float* out) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const float v = __int_as_float(speed_bits[w]);
  float dt = dt_max;
  if (v > 0.0f) dt = fminf(fmaxf(__fdiv_rn(__fmul_rn(cfl, spacing), v), dt_min), dt_max);
  out[w] = dt;
}

// Patch emitters (patch.py): triggered one-shot emitters. An entry is one world of one registration: count[e] points
// (world frame: this path has no bodies) and as many spares reserved at registration, pool[begin[e] ..].

// patch.py:65-79: arm the entries [e0, e1) whose world is flagged (int32 or bool flags [W]) and has not fired yet.
__global__ void k_patch_trigger(int e0, int e1, const void* __restrict__ flags, int is_bool,
                                const int* __restrict__ world, const int* __restrict__ fired, int* pending) {
  const int e = e0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= e1) return;
  const int w = world[e];
  const bool on = is_bool ? reinterpret_cast<const uint8_t*>(flags)[w] != 0
                          : reinterpret_cast<const int32_t*>(flags)[w] != 0;
  if (on && fired[e] == 0) pending[e] = 1;
}

// patch.py:82-107 at the end of a step, one block per entry: an armed entry's spares become liquid at its points with
// its registration's velocity (plus the zero point velocity of the world frame), their mass into the world's mass_in.
__global__ void __launch_bounds__(256) k_patch_emit(DevP P, int E, const int* __restrict__ world,
                                                    const int* __restrict__ count, const int* __restrict__ pending,
                                                    const int* __restrict__ fired, const int* __restrict__ begin,
                                                    const int* __restrict__ pool, const float* __restrict__ points,
                                                    const int* __restrict__ group, const float* __restrict__ vel,
                                                    long long* mass_in) {
  __shared__ long long sml[8];
  const int e = blockIdx.x;
  if (e >= E || pending[e] == 0 || fired[e] != 0) return;
  const float* v = vel + 3 * (size_t)group[e];
  long long in = 0;
  for (int k = threadIdx.x; k < count[e]; k += blockDim.x) {
    const size_t b = (size_t)begin[e] + k;
    const int i = pool[b];
    P.q[3 * (size_t)i] = points[3 * b];
    P.q[3 * (size_t)i + 1] = points[3 * b + 1];
    P.q[3 * (size_t)i + 2] = points[3 * b + 2];
    P.qd[3 * (size_t)i] = v[0] + 0.0f;
    P.qd[3 * (size_t)i + 1] = v[1] + 0.0f;
    P.qd[3 * (size_t)i + 2] = v[2] + 0.0f;
    P.flags[i] |= FLAG_ACTIVE;
    P.phase[i] = PH_LIQUID;
    in += to_fixed(P.mass[i]);
  }
  const long long sum = block_sum256_ll(in, sml);
  if (threadIdx.x == 0) atomicAdd((unsigned long long*)&mass_in[world[e]], (unsigned long long)sum);
}

// patch.py:110-115: an armed entry has fired; every entry is disarmed.
__global__ void k_patch_fire(int E, int* pending, int* fired) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  if (pending[e] != 0 && fired[e] == 0) fired[e] = 1;
  pending[e] = 0;
}

// patch.py:225-234 (reset): the masked worlds' entries re-armed (pending and fired cleared).
__global__ void k_patch_reset(int E, const int* __restrict__ world, const uint8_t* __restrict__ mask, int* pending,
                              int* fired) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E || !mask[world[e]]) return;
  pending[e] = 0;
  fired[e] = 0;
}

}  // namespace adf
