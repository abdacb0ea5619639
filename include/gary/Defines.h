// Scalar types and launch constants of the C++ shim layer.
//
// Same names as the reference's include/Defines.h:7-33.  Ids are unsigned
// here (vidT = uint32_t, eidT = uint64_t; the reference uses int32_t /
// int64_t): the device lists are padded with UINT32_MAX, which must sort after
// every vertex id.  For ids below 2^31 the order and arithmetic are the same.
#pragma once
#include <cstddef>
#include <cstdint>

typedef uint32_t vidT;
typedef uint64_t eidT;

constexpr int WARP_SIZE = 32;
constexpr int MAX_WARPS_PER_BLOCK = 32;
constexpr unsigned FULL_MASK = 0xFFFFFFFFu;
constexpr vidT GARY_PAD = 0xFFFFFFFFu;  // list padding in the device views

#ifndef CUDA_INLINE
#define CUDA_INLINE __forceinline__
#endif
#ifndef HOST_DEVICE
#define HOST_DEVICE __host__ __device__
#endif
#ifndef HOST_ONLY
#define HOST_ONLY __host__
#endif
#ifndef DEVICE_ONLY
#define DEVICE_ONLY __device__
#endif
