// refshim.h — host stand-ins under which the reference's own CUDA kernel
// bodies compile and run on the CPU (test infrastructure for oracle/_ref:
// the reference cannot be built as a library here, so oracle/ref/build_ref.py
// compiles the kernel bodies themselves, taken from the reference sources at
// build time, against these definitions).
//
// What is stood in for, and what each stand-in assumes:
//  * CUDA built-ins: __global__ / __device__ / __constant__ are plain host
//    code; threadIdx / blockIdx are host (thread-local) variables. run_grid()
//    runs the threads of a grid one after another: exact for kernels without
//    __syncthreads or warp intrinsics (the census transform and the
//    cross-check); atomics are plain read-modify-write. run_block_threads()
//    runs one block with one host thread per CUDA thread and __syncthreads()
//    as a barrier over them (the block-level box sums).
//  * Clu::Cuda::_CDeviceSurface (CluTec.Cuda.Base/DeviceSurface.h:139-197):
//    Read2D / Write2D / ReadPixel2D / WritePixel2D at (x, y) of a pitched
//    host buffer (surf2Dread / surf2Dwrite at byte column x * sizeof(element),
//    origin 0); an access outside the image aborts. IsInside(x, y) = inside
//    the image; IsInside(x, y, bw, bh) = at least bw columns and bh rows from
//    every edge (SImageFormat::IsInside lives in the missing CluTec.Core).
//  * Clu::Cuda::_CDeviceImage::At<P>(x, y): element (x, y) of a pitched
//    host buffer.
//  * _SDisparityConfig (missing CluTec.ImgProc/DisparityConfig.h): TPixelEx =
//    4 x uint16 with r() = channel 0, TDisp = uint16, and MapPixelPos(x, d,
//    left_to_right) = x - d or x + d (the library's own mapping; the
//    reference's pixel mapping itself stays unpinned).
#pragma once
#include <barrier>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline
#define __CUDA_HDI__ inline
#define __CUDA_DI__ inline

struct dim3 {
    unsigned x = 1, y = 1, z = 1;
    dim3() = default;
    dim3(unsigned a, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
inline thread_local dim3 threadIdx, blockIdx;
inline dim3 blockDim, gridDim;
inline std::barrier<>* g_block_barrier = nullptr;
inline void __syncthreads() { g_block_barrier->arrive_and_wait(); }

template <typename T>
inline T atomicMin(T* p, T v) {
    const T o = *p;
    if (v < o) *p = v;
    return o;
}
template <typename T>
inline T atomicMax(T* p, T v) {
    const T o = *p;
    if (v > o) *p = v;
    return o;
}

// Runs kernel(args...) for every thread of a grid, one thread at a time.
template <typename F>
inline void run_grid(dim3 grid, dim3 block, F&& kernel) {
    gridDim = grid;
    blockDim = block;
    for (unsigned bz = 0; bz < grid.z; ++bz)
        for (unsigned by = 0; by < grid.y; ++by)
            for (unsigned bx = 0; bx < grid.x; ++bx) {
                blockIdx = dim3(bx, by, bz);
                for (unsigned tz = 0; tz < block.z; ++tz)
                    for (unsigned ty = 0; ty < block.y; ++ty)
                        for (unsigned tx = 0; tx < block.x; ++tx) {
                            threadIdx = dim3(tx, ty, tz);
                            kernel();
                        }
            }
}

// Runs one block (blockIdx = b) with one host thread per CUDA thread, so
// that __syncthreads() orders the block's shared data as on the device.
template <typename F>
inline void run_block_threads(dim3 block, dim3 b, F&& kernel) {
    blockDim = block;
    const unsigned n = block.x * block.y * block.z;
    std::barrier<> bar(n);
    g_block_barrier = &bar;
    std::vector<std::thread> ts;
    ts.reserve(n);
    for (unsigned t = 0; t < n; ++t)
        ts.emplace_back([&, t] {
            blockIdx = b;
            threadIdx = dim3(t % block.x, (t / block.x) % block.y, t / (block.x * block.y));
            kernel();
        });
    for (auto& t : ts) t.join();
    g_block_barrier = nullptr;
}

namespace Clu {

enum class EPixelType { Lum };
enum class EDataType { UInt8, UInt16, UInt32 };

template <typename T>
struct SPixelLum {
    using TData = T;
    T v;
    T& r() { return v; }
    const T& r() const { return v; }
};
using TPixel_Lum_UInt8 = SPixelLum<uint8_t>;

template <EPixelType P, EDataType D>
struct CastToPixel;
template <>
struct CastToPixel<EPixelType::Lum, EDataType::UInt32> {
    using Type = SPixelLum<uint32_t>;
};

namespace Cuda {

struct _CDeviceSurface {
    unsigned char* p = nullptr;
    size_t pitch = 0;
    int w = 0, h = 0;

    bool IsInside(int x, int y) const { return x >= 0 && x < w && y >= 0 && y < h; }
    bool IsInside(int x, int y, int bw, int bh) const { return x >= bw && x < w - bw && y >= bh && y < h - bh; }

    template <typename T>
    T* at(int x, int y) const {
        if (!IsInside(x, y)) {
            std::fprintf(stderr, "refshim: surface access (%d, %d) outside %dx%d\n", x, y, w, h);
            std::abort();
        }
        return reinterpret_cast<T*>(p + size_t(y) * pitch + size_t(x) * sizeof(T));
    }
    template <typename T>
    T Read2D(int x, int y) const {
        T v;
        std::memcpy(&v, at<T>(x, y), sizeof(T));
        return v;
    }
    template <typename T>
    void Write2D(const T& v, int x, int y) {
        std::memcpy(at<T>(x, y), &v, sizeof(T));
    }
    template <typename P>
    P ReadPixel2D(int x, int y) const {
        return Read2D<P>(x, y);
    }
    template <typename P>
    void WritePixel2D(const P& v, int x, int y) {
        Write2D<P>(v, x, y);
    }
};

struct _CDeviceImage {
    unsigned char* p = nullptr;
    size_t pitch = 0;
    template <typename P>
    P& At(int x, int y) {
        return *reinterpret_cast<P*>(p + size_t(y) * pitch + size_t(x) * sizeof(P));
    }
};

struct _SDisparityConfig {
    struct TPixelEx {
        using TData = uint16_t;
        uint16_t c[4];
        uint16_t& r() { return c[0]; }
        const uint16_t& r() const { return c[0]; }
    };
    using TDisp = uint16_t;
    int MapPixelPos(int x, int d, int left_to_right) const { return left_to_right ? x - d : x + d; }
};

}  // namespace Cuda
}  // namespace Clu
