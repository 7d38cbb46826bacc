// launch.cuh -- one kernel body, two launch forms.
//
// Every kernel of the evaluation is a __device__ body whose first parameter is a VGrid
// (its block index and grid size).  launch_on<BODY, MAXT, MINB>(h.rec, grid, block, smem,
// stream, args...) runs it
//   * for one system: k_one<BODY>, an ordinary launch whose VGrid is (blockIdx.x,
//     gridDim.x), with the arguments in the kernel's parameter space;
//   * for a batch: while a handle records (h.rec set), the launch is appended to the
//     handle's Recorder instead -- the kernel instance k_many<BODY>, the grid, block,
//     shared memory and the packed arguments -- and the batch later issues ONE launch of
//     k_many per stage for all its systems (csrc/batch.cu): the blocks of system s are
//     the consecutive range [pre[s], pre[s + 1]) of one grid, each reading system s's
//     packed arguments and seeing the VGrid of its own launch.
// The body cannot tell the two forms apart.  Bodies whose batch instance ran short of
// registers take their arguments by const reference: that instance then reads each one
// from the staged pack in shared memory where it is used, instead of holding them all in
// registers from the start (the single-system instance reads the parameter bank either way).  (Floating-point arithmetic whose rounding
// must not depend on the instance -- the compiler may fuse a multiply and an add in one
// instance and not in the other -- is written with explicit roundings, xmul / xadd / xfma.)
#pragma once

#include <cstring>
#include <vector>

namespace ffx {

struct VGrid {
  int bid;    // this block's index within the system's grid
  int nblk;   // the system's grid size
};

// Kernel arguments packed as a plain aggregate (trivially copyable: it is copied to the
// device as bytes).  Pack<A0, A1, ...> holds A0 first.
template <typename... A>
struct Pack;
template <>
struct Pack<> {};
template <typename H, typename... T>
struct Pack<H, T...> {
  H h;
  Pack<T...> t;
};

inline Pack<> make_pack() { return {}; }
template <typename H, typename... T>
inline Pack<H, T...> make_pack(const H &h, const T &...t) {
  Pack<H, T...> p;
  p.h = h;
  p.t = make_pack(t...);
  return p;
}

// BODY(g, a0, a1, ...) from a Pack in memory: the arguments are passed as references into
// the pack, so structures indexed at run time are read in place.
template <auto BODY, typename... D>
__device__ __forceinline__ void call_pack(const Pack<> &, VGrid g, const D &...d) {
  BODY(g, d...);
}
template <auto BODY, typename H, typename... T, typename... D>
__device__ __forceinline__ void call_pack(const Pack<H, T...> &p, VGrid g, const D &...d) {
  call_pack<BODY>(p.t, g, d..., p.h);
}

// One system.  __grid_constant__ keeps structure arguments in parameter space.  The
// launch bounds are the body's own: (MAXT, MINB); MINB = 0 gives __launch_bounds__(MAXT)
// alone and MAXT = 0 none (each choice changes how the compiler allocates registers).
template <auto BODY, int MAXT, int MINB, typename... A>
__global__ void __launch_bounds__(MAXT, MINB) k_one(const __grid_constant__ A... a) {
  BODY(VGrid{(int)blockIdx.x, (int)gridDim.x}, a...);
}
template <auto BODY, int MAXT, typename... A>
__global__ void __launch_bounds__(MAXT) k_one_max(const __grid_constant__ A... a) {
  BODY(VGrid{(int)blockIdx.x, (int)gridDim.x}, a...);
}
template <auto BODY, typename... A>
__global__ void k_one_free(const __grid_constant__ A... a) {
  BODY(VGrid{(int)blockIdx.x, (int)gridDim.x}, a...);
}

// Every system of a batch in one grid.  pre[0 .. ns] are the systems' first blocks
// (pre[ns] = the grid); loop_cont, when set, is each system's solver flag (PcgState::cont):
// launches inside the solver's loop skip systems whose solve has stopped.  The system's
// arguments are staged in shared memory, where the body reads them as it uses them
// (held in registers from the start they raise the register count).
template <auto BODY, typename... A>
__device__ __forceinline__ void many_body(const Pack<A...> *__restrict__ args, const int *__restrict__ pre,
                                          const int *const *__restrict__ loop_cont, int ns) {
  const int b = (int)blockIdx.x;
  int lo = 0, hi = ns;
  while (hi - lo > 1) {
    const int m = (lo + hi) >> 1;
    if (pre[m] <= b) lo = m;
    else hi = m;
  }
  if (loop_cont && !*loop_cont[lo]) return;
  __shared__ __align__(16) unsigned char sp[sizeof(Pack<A...>)];
  const unsigned *src = reinterpret_cast<const unsigned *>(args + lo);
  for (int w = threadIdx.x; w < (int)(sizeof(Pack<A...>) / 4); w += blockDim.x)
    reinterpret_cast<unsigned *>(sp)[w] = src[w];
  __syncthreads();
  call_pack<BODY>(*reinterpret_cast<const Pack<A...> *>(sp), VGrid{b - pre[lo], pre[lo + 1] - pre[lo]});
}
template <auto BODY, int MAXT, int MINB, typename... A>
__global__ void __launch_bounds__(MAXT, MINB)
    k_many(const Pack<A...> *__restrict__ args, const int *__restrict__ pre, const int *const *__restrict__ loop_cont,
           int ns) {
  many_body<BODY>(args, pre, loop_cont, ns);
}
template <auto BODY, int MAXT, typename... A>
__global__ void __launch_bounds__(MAXT)
    k_many_max(const Pack<A...> *__restrict__ args, const int *__restrict__ pre, const int *const *__restrict__ loop_cont,
               int ns) {
  many_body<BODY>(args, pre, loop_cont, ns);
}
template <auto BODY, typename... A>
__global__ void k_many_free(const Pack<A...> *__restrict__ args, const int *__restrict__ pre,
                            const int *const *__restrict__ loop_cont, int ns) {
  many_body<BODY>(args, pre, loop_cont, ns);
}

// A body as a type, for launch sites that choose among template instances at run time.
template <auto F>
struct BodyOf {
  static constexpr auto value = F;
};

// One recorded launch of a system.
struct RecLaunch {
  const void *fn = nullptr;        // the k_many instance (identifies the stage's kernel)
  int grid = 0, block = 0;
  size_t smem = 0;
  std::vector<unsigned char> pack; // the packed arguments
  int phase = 0;                   // 0 before the solver's loop, 1 inside it, 2 after it
};

// A system's evaluation as recorded launches, plus its device-to-host result copies,
// which the batch gathers into one staging buffer (source, offset in the system's staging
// slot, host destination, bytes).
struct Recorder {
  std::vector<RecLaunch> seq;
  int phase = 0;
  struct Copy {
    const void *src;
    size_t off;
    void *host;
    size_t bytes;
  };
  std::vector<Copy> copies;
  size_t stage_bytes = 0;
};

// The single-system and batch kernel instances of a body with arguments A... (for
// cudaFuncSetAttribute; the address is taken where BODY is a template parameter).
template <auto BODY, int MAXT, int MINB, typename... A>
inline const void *one_fn() {
  if constexpr (MAXT == 0) return (const void *)k_one_free<BODY, A...>;
  else if constexpr (MINB == 0) return (const void *)k_one_max<BODY, MAXT, A...>;
  else return (const void *)k_one<BODY, MAXT, MINB, A...>;
}
template <auto BODY, int MAXT, int MINB, typename... A>
inline const void *many_fn() {
  if constexpr (MAXT == 0) return (const void *)k_many_free<BODY, A...>;
  else if constexpr (MINB == 0) return (const void *)k_many_max<BODY, MAXT, A...>;
  else return (const void *)k_many<BODY, MAXT, MINB, A...>;
}

// MB: the batch instance's minimum resident blocks (0: the single-system bounds).  A
// batch kernel reads its arguments from memory, not from the parameter bank, and keeps
// them in registers; MB caps the registers where that would cost occupancy.
template <auto BODY, int MAXT, int MINB, int MB = MINB, typename... A>
inline void launch_on(Recorder *rec, int grid, int block, size_t smem, cudaStream_t st, const A &...a) {
  if (rec) {
    RecLaunch r;
    r.fn = many_fn<BODY, MAXT, MB, A...>();
    r.grid = grid;
    r.block = block;
    r.smem = smem;
    const Pack<A...> p = make_pack(a...);
    r.pack.resize(sizeof(p));
    std::memcpy(r.pack.data(), &p, sizeof(p));
    r.phase = rec->phase;
    rec->seq.push_back(std::move(r));
    return;
  }
  if constexpr (MAXT == 0) k_one_free<BODY, A...><<<grid, block, smem, st>>>(a...);
  else if constexpr (MINB == 0) k_one_max<BODY, MAXT, A...><<<grid, block, smem, st>>>(a...);
  else k_one<BODY, MAXT, MINB, A...><<<grid, block, smem, st>>>(a...);
}

}  // namespace ffx
