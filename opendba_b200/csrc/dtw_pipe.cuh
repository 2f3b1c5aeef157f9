// Bounded hand-off of swath-edge rows between warps (the swath pipeline).
//
// The producing warp's lane 31 publishes "rows stored so far" with a
// gpu-scope release; the consuming warp's lane 0 acquires the word before it
// reads rows it has not seen published.  Every wait is bounded: after the
// limit (%globaltimer) the waiter raises the launch's error word and goes on,
// and every other waiter that sees the word stops waiting too.
#pragma once

#include <cstdint>

namespace odba {

constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_timer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct PipeGate {
  static constexpr bool kActive = true;
  const unsigned long long *prog_in;  // progress word of the previous swath
  unsigned long long *prog_out;       // progress word of this swath
  unsigned *err;
  unsigned long long limit_ns;
  int avail;                          // input rows known to be published

  __device__ __forceinline__ void wait_in(int k) {
    if (k <= avail) return;
    unsigned long long t0 = 0;
    for (unsigned it = 0;; ++it) {
      const unsigned long long v = ld_acquire_gpu(prog_in);
      if (v >= (unsigned long long)k) {
        avail = int(v);
        return;
      }
      if (*reinterpret_cast<volatile unsigned *>(err)) {
        avail = 0x7fffffff;
        return;
      }
      const unsigned long long now = global_timer_ns();
      if (it == 0) {
        t0 = now;
      } else if (now - t0 > limit_ns) {
        atomicExch(err, 1u);
        avail = 0x7fffffff;
        return;
      }
      __nanosleep(128);
    }
  }
  __device__ __forceinline__ void publish(int k) { st_release_gpu(prog_out, (unsigned long long)k); }
};

// The gate of a band of a swath's rows: the band's rows count from base (its
// first row's offset in the swath), so the progress words keep counting the
// whole swath's rows whichever band publishes them.
struct BandGate {
  static constexpr bool kActive = true;
  PipeGate g;
  int base;
  __device__ __forceinline__ void wait_in(int k) { g.wait_in(base + k); }
  __device__ __forceinline__ void publish(int k) { g.publish(base + k); }
};

// Bounded wait (one thread) until *p >= v, with the gate's error rules:
// false if the limit ran out (the error word is raised) or another waiter
// raised it.
__device__ __forceinline__ bool wait_word_at_least(const unsigned long long *p, unsigned long long v,
                                                   unsigned *err, unsigned long long limit_ns) {
  unsigned long long t0 = 0;
  for (unsigned it = 0;; ++it) {
    if (ld_acquire_gpu(p) >= v) return true;
    if (*reinterpret_cast<volatile unsigned *>(err)) return false;
    const unsigned long long now = global_timer_ns();
    if (it == 0) {
      t0 = now;
    } else if (now - t0 > limit_ns) {
      atomicExch(err, 1u);
      return false;
    }
    __nanosleep(128);
  }
}

}  // namespace odba
