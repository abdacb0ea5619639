// Byte planes: split an array of 4- or 8-byte words into planes of 1, 2 or 4
// bytes (plane j holds byte group j of every word, least significant first),
// and join them back.  The reference's segmentKernel<SrcT, DstT>
// (include/kernels/SegmentArray.cuh:26-149) does the split through shared
// memory with cooperative-groups memcpy_async, as a bandwidth experiment for
// compressible adjacency (high-order planes of sorted ids repeat).
//
// Here the transform is a pure HBM stream with no shared memory: each thread
// takes a group of G = 16 / plane_bytes words, loads them with 16-byte loads,
// and writes every plane's G entries as one 16-byte store; grids are sized to
// the SM count and stride over the groups.  Pointers must be 16-byte aligned
// (cudaMalloc's are); words past the last whole group go through a scalar
// tail.  Both directions move n * src_bytes bytes each way.
#include "internal.cuh"

namespace gary {
namespace {

constexpr int kPlThreads = 256;

template <int SB, int PB>
struct PlaneGeom {
  static constexpr int K = SB / PB;         // planes
  static constexpr int G = 16 / PB;         // words per thread group
  static constexpr int SRC_VEC = G * SB / 16;  // 16-byte loads of source per group
};

struct PlanePtrs {
  uint8_t *p[8];
};

template <int SB, int PB>
__global__ void __launch_bounds__(kPlThreads) k_split(const uint8_t *__restrict__ src, uint64_t n,
                                                      PlanePtrs planes) {
  using Geo = PlaneGeom<SB, PB>;
  const uint64_t groups = n / Geo::G;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < groups; g += stride) {
    union {
      uint4 v[Geo::SRC_VEC];
      uint8_t b[Geo::G * SB];
    } in;
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src + g * Geo::G * SB);
#pragma unroll
    for (int k = 0; k < Geo::SRC_VEC; ++k) in.v[k] = s4[k];
#pragma unroll
    for (int j = 0; j < Geo::K; ++j) {
      union {
        uint4 v;
        uint8_t b[16];
      } out;
#pragma unroll
      for (int w = 0; w < Geo::G; ++w)
#pragma unroll
        for (int c = 0; c < PB; ++c) out.b[w * PB + c] = in.b[w * SB + j * PB + c];
      reinterpret_cast<uint4 *>(planes.p[j])[g] = out.v;
    }
  }
  // tail: the words after the last whole group, one per thread
  const uint64_t t0 = groups * Geo::G;
  for (uint64_t i = t0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
#pragma unroll
    for (int j = 0; j < Geo::K; ++j)
#pragma unroll
      for (int c = 0; c < PB; ++c) planes.p[j][i * PB + c] = src[i * SB + j * PB + c];
}

template <int SB, int PB>
__global__ void __launch_bounds__(kPlThreads) k_join(PlanePtrs planes, uint64_t n,
                                                     uint8_t *__restrict__ dst) {
  using Geo = PlaneGeom<SB, PB>;
  const uint64_t groups = n / Geo::G;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < groups; g += stride) {
    union {
      uint4 v[Geo::SRC_VEC];
      uint8_t b[Geo::G * SB];
    } out;
#pragma unroll
    for (int j = 0; j < Geo::K; ++j) {
      union {
        uint4 v;
        uint8_t b[16];
      } in;
      in.v = reinterpret_cast<const uint4 *>(planes.p[j])[g];
#pragma unroll
      for (int w = 0; w < Geo::G; ++w)
#pragma unroll
        for (int c = 0; c < PB; ++c) out.b[w * SB + j * PB + c] = in.b[w * PB + c];
    }
    uint4 *d4 = reinterpret_cast<uint4 *>(dst + g * Geo::G * SB);
#pragma unroll
    for (int k = 0; k < Geo::SRC_VEC; ++k) d4[k] = out.v[k];
  }
  const uint64_t t0 = groups * Geo::G;
  for (uint64_t i = t0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
#pragma unroll
    for (int j = 0; j < Geo::K; ++j)
#pragma unroll
      for (int c = 0; c < PB; ++c) dst[i * SB + j * PB + c] = planes.p[j][i * PB + c];
}

unsigned plane_grid(uint64_t items) {
  const uint64_t b = (items + kPlThreads - 1) / kPlThreads;
  const uint64_t cap = (uint64_t)sm_count() * 8;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <bool SPLIT, int SB, int PB>
int launch_planes(uint8_t *words, uint64_t n, const PlanePtrs &pp, cudaStream_t s) {
  using Geo = PlaneGeom<SB, PB>;
  const uint64_t items = n / Geo::G + (n % Geo::G ? 1 : 0);
  if (SPLIT) k_split<SB, PB><<<plane_grid(items), kPlThreads, 0, s>>>(words, n, pp);
  else k_join<SB, PB><<<plane_grid(items), kPlThreads, 0, s>>>(pp, n, words);
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

template <bool SPLIT>
int planes_dispatch(uint8_t *words, uint64_t n, int sb, int pb, const PlanePtrs &pp, cudaStream_t s) {
  if (sb == 4 && pb == 1) return launch_planes<SPLIT, 4, 1>(words, n, pp, s);
  if (sb == 4 && pb == 2) return launch_planes<SPLIT, 4, 2>(words, n, pp, s);
  if (sb == 8 && pb == 1) return launch_planes<SPLIT, 8, 1>(words, n, pp, s);
  if (sb == 8 && pb == 2) return launch_planes<SPLIT, 8, 2>(words, n, pp, s);
  if (sb == 8 && pb == 4) return launch_planes<SPLIT, 8, 4>(words, n, pp, s);
  set_error("word/plane sizes %d/%d not supported (4/1, 4/2, 8/1, 8/2, 8/4)", sb, pb);
  return GARY_ERR_INVALID;
}

int planes_args(const void *words, void *const *planes, uint64_t n, int sb, int pb, PlanePtrs &pp) {
  GARY_CHECK_ARG((sb == 4 || sb == 8) && (pb == 1 || pb == 2 || pb == 4) && pb < sb,
                 "word/plane sizes %d/%d not supported", sb, pb);
  GARY_CHECK_ARG(n == 0 || (words && planes), "NULL argument");
  GARY_CHECK_ARG(n == 0 || aligned16(words), "the word array must be 16-byte aligned");
  if (n == 0) return GARY_OK;
  for (int j = 0; j < sb / pb; ++j) {
    GARY_CHECK_ARG(planes[j] && aligned16(planes[j]), "plane %d is NULL or not 16-byte aligned", j);
    pp.p[j] = static_cast<uint8_t *>(planes[j]);
  }
  return GARY_OK;
}

}  // namespace
}  // namespace gary

extern "C" int gary_planes_split(const void *d_words, uint64_t n, int word_bytes, int plane_bytes,
                                 void *const *d_planes, void *stream) {
  gary::PlanePtrs pp{};
  GARY_TRY(gary::planes_args(d_words, d_planes, n, word_bytes, plane_bytes, pp));
  if (!n) return GARY_OK;
  return gary::planes_dispatch<true>(const_cast<uint8_t *>(static_cast<const uint8_t *>(d_words)), n,
                                     word_bytes, plane_bytes, pp, gary::as_stream(stream));
}

extern "C" int gary_planes_join(void *const *d_planes, uint64_t n, int word_bytes, int plane_bytes,
                                void *d_words, void *stream) {
  gary::PlanePtrs pp{};
  GARY_TRY(gary::planes_args(d_words, d_planes, n, word_bytes, plane_bytes, pp));
  if (!n) return GARY_OK;
  return gary::planes_dispatch<false>(static_cast<uint8_t *>(d_words), n, word_bytes, plane_bytes, pp,
                                      gary::as_stream(stream));
}
