// walk_kernels.cuh -- the walk kernels and their launch dispatch, shared by
// the translation units that instantiate them (walk_*.cu; one output kind or
// reduction family each, so the kernels compile in parallel) and by
// project.cu (host logic, diagnosis, scatter and sampling kernels).
//
// Sinks: the fused reductions of src/reduction.cpp:8-96, the CSR segment
// writer of src/projection.cpp:75-144, the segment tape and the adjoint
// scatter.  Kernels: k_plain (one ray per thread, exact FP64 search from the
// root for every query: the straightforward port and the baseline kernel),
// k_slow (finishes handed-over rays with a global-memory pending-point
// stack), k_batched (batched.cuh) and k_warp (warp.cuh).
#pragma once

#include <type_traits>

#include "internal.h"
#include "walk.cuh"
#include "walkio.h"

namespace vt {

constexpr int kPlainStack = 48;

__device__ __forceinline__ double pinf() { return __longlong_as_double(0x7ff0000000000000LL); }

// ------------------------------------------------------------------ sinks
// Fused reduction in segment order (src/reduction.cpp:8-83).  NF > 0: the
// field count known at compile time, accumulators in registers; NF == 0: any
// count, accumulated in place in the output row.
template <int MODE, int NF>
struct Reducer {
  const DevCloud* c;
  double* row;
  double acc[NF > 0 ? NF : 3];
  double T;
  unsigned nseg;
  __device__ __forceinline__ void init(const DevCloud* cc, double* r) {
    c = cc;
    row = r;
    nseg = 0;
    T = 1.0;
    const double init = MODE == kMax ? -pinf() : (MODE == kMin ? pinf() : 0.0);
    if (MODE == kVolume) {
      acc[0] = acc[1] = acc[2] = 0.0;
    } else if (NF > 0) {
#pragma unroll
      for (int f = 0; f < (NF > 0 ? NF : 1); ++f) acc[f] = init;
    } else {
      for (int f = 0; f < c->nf; ++f) row[f] = init;
    }
  }
  __device__ __forceinline__ void seg(int cell, double a, double b) {
    ++nseg;
    const int nf = NF > 0 ? NF : c->nf;
    const double* F = c->fields + (int64_t)cell * nf;
    if (MODE == kVolume) {
      // reduce_volume_render (src/reduction.cpp:68-80)
      const double alpha = F[3];
      const double ds = dsub(b, a);
      const double opac = dsub(1.0, exp(dmul(-alpha, ds)));
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[k] = dadd(acc[k], dmul(dmul(T, F[k]), opac));
      T = dmul(T, dsub(1.0, opac));
    } else if (NF > 0) {
      const double ds = dsub(b, a);
#pragma unroll
      for (int f = 0; f < (NF > 0 ? NF : 1); ++f) {
        const double v = F[f];
        if (MODE == kSum) acc[f] = dadd(acc[f], dmul(ds, v));
        else if (MODE == kMax) acc[f] = v > acc[f] ? v : acc[f];
        else acc[f] = v < acc[f] ? v : acc[f];
      }
    } else {
      const double ds = dsub(b, a);
      for (int f = 0; f < nf; ++f) {
        const double v = F[f];
        if (MODE == kSum) row[f] = dadd(row[f], dmul(ds, v));
        else if (MODE == kMax) row[f] = v > row[f] ? v : row[f];
        else row[f] = v < row[f] ? v : row[f];
      }
    }
  }
  __device__ __forceinline__ void write(double* out) const {
    if (MODE == kVolume) {
      out[0] = acc[0];
      out[1] = acc[1];
      out[2] = acc[2];
    } else if (NF > 0) {
#pragma unroll
      for (int f = 0; f < (NF > 0 ? NF : 1); ++f) out[f] = acc[f];
    }
  }
};

// Append one tape entry; the lanes of a warp that reach this point together
// reserve their slots with one atomic.  Entries past tape_cap are counted
// but not written (the host then sizes the tape from the count).
// Append one tape entry from one lane (its own slot).  Entries past
// tape_cap are counted but not written (the host then sizes the tape from
// the count).
template <class E>
__device__ __forceinline__ void tape_append(const WalkIO& io, const E& e) {
  const unsigned long long k = atomicAdd(io.tape_count, 1ULL);
  if (k < io.tape_cap) static_cast<E*>(io.tape)[k] = e;
}

// Reducer of 'integrate' or 'volume' that also records the tape; the first
// `skip` segments of the ray were recorded by an earlier, handed-over launch.
// STAGED (the batched thread kernel): the segments of one loop trip (at most
// two) wait in registers and flush_tape, which every lane of the warp calls
// at the end of each trip, writes them with one atomic per warp; otherwise
// each segment takes its own slot.
template <int MODE, int NF, bool STAGED = false>
struct TapeReducer : Reducer<MODE, NF> {
  using E = typename std::conditional<MODE == kVolume, TapeEntryV, TapeEntry>::type;
  const WalkIO* io;
  int ray;
  unsigned skip;
  int npend = 0;
  E pend[2];
  __device__ __forceinline__ void set_tape(const WalkIO* w, int64_t r, unsigned sk) {
    io = w;
    ray = (int)r;
    skip = sk;
  }
  __device__ __forceinline__ void record(const E& e) {
    if (STAGED) {
      if (npend == 0) pend[0] = e;
      else pend[1] = e;
      ++npend;
    } else {
      tape_append(*io, e);
    }
  }
  __device__ __forceinline__ void seg(int cell, double a, double b) {
    if constexpr (MODE == kVolume) {
      const double T0 = this->T;
      Reducer<MODE, NF>::seg(cell, a, b);
      if (this->nseg > skip)
        record(TapeEntryV{cell, ray, dsub(b, a), T0, {this->acc[0], this->acc[1], this->acc[2]}});
    } else {
      Reducer<MODE, NF>::seg(cell, a, b);
      if (this->nseg > skip) record(TapeEntry{this->c->perm[cell], ray, dsub(b, a)});
    }
  }
  // all 32 lanes: write the staged entries (warp prefix sum, one atomic)
  __device__ __forceinline__ void flush_tape(const WalkIO& w) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int incl = npend;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(full, incl, 31);
    if (total == 0) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(w.tape_count, (unsigned long long)total);
    base = __shfl_sync(full, base, 0);
    const unsigned long long k = base + (unsigned long long)(incl - npend);
    E* t = static_cast<E*>(w.tape);
    if (npend > 0 && k < w.tape_cap) t[k] = pend[0];
    if (npend > 1 && k + 1 < w.tape_cap) t[k + 1] = pend[1];
    npend = 0;
  }
};

// CSR segment writer (src/projection.cpp:221-238): internal ids via perm.
struct FillSink {
  const DevCloud* c;
  int64_t* cell;
  double* se;
  double* sx;
  int64_t off;
  unsigned nseg;
  __device__ __forceinline__ void init(const DevCloud* cc, const WalkIO& io, int64_t ray) {
    c = cc;
    cell = io.seg_cell;
    se = io.seg_enter;
    sx = io.seg_exit;
    off = io.offsets[ray];
    nseg = 0;
  }
  __device__ __forceinline__ void seg(int cl, double a, double b) {
    const int64_t k = off + nseg;
    cell[k] = c->perm[cl];
    se[k] = a;
    sx[k] = b;
    ++nseg;
  }
};

// Adjoint of the reductions w.r.t. the per-cell fields.  The first `skip`
// segments were already scattered by an earlier, handed-over launch.
//   SUM:    g[c,f] += gbar[f] * ds
//   VOLUME: o = 1 - exp(-alpha ds), T transmittance before the segment,
//           S = sum of later contributions = C - (prefix incl. this one)
//           d/d rgb_k   = gbar_k T o
//           d/d alpha   = ds * sum_k gbar_k (T rgb_k (1 - o) - S_k)
template <int MODE, int NF>
struct AdjSink {
  const DevCloud* c;
  double* grad;
  const double* grow;  // upstream gradient row
  double g[NF > 0 ? NF : 3];
  double C[3], P[3];
  double T;
  unsigned nseg, skip;
  __device__ __forceinline__ void init(const DevCloud* cc, const WalkIO& io, int64_t ray,
                                       unsigned sk) {
    c = cc;
    grad = io.grad;
    grow = io.gout + ray * io.nout;
    skip = sk;
    nseg = 0;
    T = 1.0;
    if (MODE == kVolume) {
      for (int k = 0; k < 3; ++k) {
        g[k] = grow[k];
        C[k] = io.fwd[ray * 3 + k];
        P[k] = 0.0;
      }
    } else if (NF > 0) {
#pragma unroll
      for (int f = 0; f < (NF > 0 ? NF : 1); ++f) g[f] = grow[f];
    }
  }
  __device__ __forceinline__ void seg(int cell, double a, double b) {
    const bool emit = nseg >= skip;
    ++nseg;
    const double ds = dsub(b, a);
    const int nf = NF > 0 ? NF : c->nf;
    const int64_t pid = c->perm[cell];
    if (MODE == kVolume) {
      const double* F = c->fields + (int64_t)cell * 4;
      const double alpha = F[3];
      const double e = exp(dmul(-alpha, ds));
      const double o = dsub(1.0, e);
      double galpha = 0.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double contrib = dmul(dmul(T, F[k]), o);
        P[k] = dadd(P[k], contrib);
        const double S = C[k] - P[k];
        galpha += g[k] * (T * F[k] * e - S);
        if (emit) atomicAdd(&grad[pid * 4 + k], g[k] * T * o);
      }
      if (emit) atomicAdd(&grad[pid * 4 + 3], ds * galpha);
      T = dmul(T, dsub(1.0, o));  // same rounding as the forward pass
    } else if (NF > 0) {
      if (emit) {
#pragma unroll
        for (int f = 0; f < (NF > 0 ? NF : 1); ++f) atomicAdd(&grad[pid * nf + f], g[f] * ds);
      }
    } else if (emit) {
      for (int f = 0; f < nf; ++f) atomicAdd(&grad[pid * nf + f], grow[f] * ds);
    }
  }
};

struct NullSink {
  unsigned nseg = 0;
  __device__ __forceinline__ void seg(int, double, double) { ++nseg; }
};

// ------------------------------------------------------- per-ray driver
template <int MODE, int NF, int OUT, class Srch, class Stack>
__device__ __forceinline__ int run_ray(const DevCloud& c, const WalkIO& io, int64_t ray,
                                       Srch& S, Stack& st, unsigned skip, unsigned& nseg) {
  RayGeom g;
  ray_init(g, io.starts + 3 * ray, io.ends + 3 * ray);
  if (!ray_finite(g)) {
    nseg = 0;
    return kErrNonFinite;
  }
  int rc;
  if (OUT == kOutImage || OUT == kOutCount) {
    double* row = io.out + ray * io.nout;
    Reducer<MODE, NF> red;
    red.init(&c, row);
    rc = walk_ray(c, g, io.max_iter, S, st, red, (WalkDiag*)nullptr);
    nseg = red.nseg;
    if (rc == 0) {
      red.write(row);
      if (OUT == kOutCount) io.counts[ray] = red.nseg;
    }
  } else if (OUT == kOutTape) {
    double* row = io.out + ray * io.nout;
    TapeReducer<MODE, NF> red;
    red.init(&c, row);
    red.set_tape(&io, ray, skip);
    rc = walk_ray(c, g, io.max_iter, S, st, red, (WalkDiag*)nullptr);
    nseg = red.nseg;
    if (rc == 0) red.write(row);
  } else if (OUT == kOutFill) {
    FillSink fs;
    fs.init(&c, io, ray);
    rc = walk_ray(c, g, io.max_iter, S, st, fs, (WalkDiag*)nullptr);
    nseg = fs.nseg;
  } else {
    AdjSink<MODE, NF> as;
    as.init(&c, io, ray, skip);
    rc = walk_ray(c, g, io.max_iter, S, st, as, (WalkDiag*)nullptr);
    nseg = as.nseg;
  }
  return rc;
}

__device__ __forceinline__ void report(const WalkIO& io, int64_t ray, int rc) {
  if (rc && rc != kNeedSlow && rc != kNeedTie)
    atomicMin(&io.stats->first_error, ((unsigned long long)ray << 8) | (unsigned)rc);
}

__device__ __forceinline__ void hand_over(const WalkIO& io, int64_t ray, unsigned emitted) {
  const unsigned long long k = atomicAdd(&io.stats->slow_count, 1ULL);
  io.slow_q[k] = ((unsigned long long)ray << 24) | (emitted & 0xffffffu);
}

// ------------------------------------------------------------ k_plain
template <int MODE, int NF, int OUT, bool PER>
__global__ void __launch_bounds__(128) k_plain(DevCloud c, WalkIO io) {
  const int64_t ray = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (ray >= io.nrays) return;
  Search64T<PER> S(c);
  LocalStack<kPlainStack> st;
  st.set_cap(io.local_cap);
  st.clear();
  unsigned nseg = 0;
  int rc = run_ray<MODE, NF, OUT>(c, io, ray, S, st, 0u, nseg);
  if (rc == kNeedSlow || rc == kNeedTie) hand_over(io, ray, nseg);
  report(io, ray, rc);
  warp_add(&io.stats->rays, 1u);
  warp_add(&io.stats->crossings, rc == 0 ? nseg : 0u);
  warp_add(&io.stats->queries, S.nq);
  warp_max(&io.stats->max_stack, (unsigned)st.maxsp);
}

// hand-over queue entries: ray in bits 24-62, segments already emitted in
// bits 0-23; bit 63 marks a ray deferred until the reference-order tree
// exists
constexpr unsigned long long kDeferredBit = 1ULL << 63;
__device__ __forceinline__ int64_t queued_ray(unsigned long long e) {
  return (int64_t)((e & ~kDeferredBit) >> 24);
}

// ------------------------------------------------------------- k_slow
// Finishes the handed-over rays.  A ray whose 1-NN query meets an exact tie
// while the reference-order tree is not built yet is deferred: its queue
// entry is marked (with the segments emitted up to the tie, all of them the
// reference's) and the host builds the tree and runs this kernel again with
// io.deferred set, over the marked entries only.
template <int MODE, int NF, int OUT, bool PER>
__global__ void __launch_bounds__(128) k_slow(DevCloud c, WalkIO io) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  GlobalStack st;
  st.id = io.gstack_id + (int64_t)tid * io.gstack_cap;
  st.s = io.gstack_s + (int64_t)tid * io.gstack_cap;
  st.cap = io.gstack_cap;
  st.clear();
  const unsigned long long total = io.stats->slow_count;
  for (unsigned long long q = tid; q < total; q += io.slow_threads) {
    const unsigned long long e = io.slow_q[q];
    if (io.deferred && !(e & kDeferredBit)) continue;
    const int64_t ray = queued_ray(e);
    const unsigned skip = (unsigned)(e & 0xffffffu);
    Search64T<PER, true> S(c);
    unsigned nseg = 0;
    int rc = run_ray<MODE, NF, OUT>(c, io, ray, S, st, skip, nseg);
    if (rc == kNeedSlow) rc = kErrStack;
    if (rc == kNeedTie && !io.deferred) {
      io.slow_q[q] = kDeferredBit | ((unsigned long long)ray << 24) | (nseg & 0xffffffu);
      atomicAdd(&io.stats->tie_deferred, 1ULL);
    } else {
      if (rc == kNeedTie) rc = kErrTie;
      report(io, ray, rc);
      if (rc == 0) atomicAdd(&io.stats->crossings, (unsigned long long)nseg);
      if (S.nties) atomicAdd(&io.stats->ties, (unsigned long long)S.nties);
    }
    if (!io.deferred) atomicAdd(&io.stats->slow_rays, 1ULL);
    atomicAdd(&io.stats->queries, (unsigned long long)S.nq);
    atomicMax(&io.stats->max_stack, (unsigned long long)st.maxsp);
  }
}


}  // namespace vt

// persistent kernels: one ray per thread (batched.cuh), one ray per warp
// with warp-cooperative search (warp.cuh)
#include "batched.cuh"
#include "warp.cuh"

namespace vt {

// ------------------------------------------------------------ dispatch
template <int MODE, int NF, int OUT>
int launch_walk_t(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st) {
  const DevCloud& c = cl->view;
  if (io.nrays > 0) {
    const int B = 128;
    if (io.deferred) {
      // second pass over the rays deferred for the reference-order tree
    } else if (cl->periodic) {
      k_plain<MODE, NF, OUT, true><<<(unsigned)((io.nrays + B - 1) / B), B, 0, st>>>(c, io);
    } else if (kernel == VT_KERNEL_PLAIN_FP64) {
      k_plain<MODE, NF, OUT, false><<<(unsigned)((io.nrays + B - 1) / B), B, 0, st>>>(c, io);
    } else if (kernel == VT_KERNEL_BATCHED && cl->nfields <= 32) {
      int rc = launch_warp<MODE, OUT>(cl, io, st);
      if (rc) return rc;
    } else {
      int rc = launch_batched<MODE, NF, OUT>(cl, io, kernel, st);
      if (rc) return rc;
    }
    VT_CUDA(cudaGetLastError());
    const int SB = 128;
    if (cl->periodic)
      k_slow<MODE, NF, OUT, true><<<(unsigned)(io.slow_threads / SB), SB, 0, st>>>(c, io);
    else
      k_slow<MODE, NF, OUT, false><<<(unsigned)(io.slow_threads / SB), SB, 0, st>>>(c, io);
    VT_CUDA(cudaGetLastError());
  }
  return VT_OK;
}

// 'integrate' with the field count known at compile time for 1, 3 and 4
// fields (accumulators in registers), any other count accumulated in place
template <int OUT>
int launch_sum(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st) {
  switch ((int)cl->nfields) {
    case 1: return launch_walk_t<kSum, 1, OUT>(cl, io, kernel, st);
    case 3: return launch_walk_t<kSum, 3, OUT>(cl, io, kernel, st);
    case 4: return launch_walk_t<kSum, 4, OUT>(cl, io, kernel, st);
    default: return launch_walk_t<kSum, 0, OUT>(cl, io, kernel, st);
  }
}

// 'volume', 'max' and 'min'
template <int OUT>
int launch_vmm(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st) {
  const bool one = cl->nfields == 1;
  if (mode == kVolume) return launch_walk_t<kVolume, 4, OUT>(cl, io, kernel, st);
  if (mode == kMax)
    return one ? launch_walk_t<kMax, 1, OUT>(cl, io, kernel, st)
               : launch_walk_t<kMax, 0, OUT>(cl, io, kernel, st);
  return one ? launch_walk_t<kMin, 1, OUT>(cl, io, kernel, st)
             : launch_walk_t<kMin, 0, OUT>(cl, io, kernel, st);
}

}  // namespace vt
