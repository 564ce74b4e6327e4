// Host harness for elsa's own CUDA projector kernels, so that they can be timed on the same GPU as
// this library's kernels. TEST INFRASTRUCTURE ONLY (tests/ load it); nothing in the elsa_b200
// package uses it.
//
// The kernels are compiled from the reference's sources where they lie
// (projectors_cuda/projector_kernels/TraverseJosephsCUDA.cu, TraverseSiddonsCUDA.cu,
// ProjectVoxelsCUDA.cu) with the stand-in headers in shim/. This file sets up the buffers the
// reference's operators hand to those kernels, written from their documented layouts:
//   * JosephsMethodCUDA.cpp:9-91: ray origins (pitched, dim floats per pose), the inverse and the
//     plain projection matrices' top-left dim x dim blocks (cudaMalloc3D, one matrix column per
//     pitched row); forward: the volume as a linear-filtered, clamped 3D texture and a pitched
//     sinogram (:120-214); the default `fast` adjoint: the sinogram as a layered, border-addressed
//     2D texture and a pitched volume (:216-259).
//   * SiddonsMethodCUDA.cpp:30-58,104-210: dense column-major inverse blocks and camera centres;
//     dense volume and sinogram, zeroed before the kernels accumulate.
//   * VoxelCUDAHelper.cuh:18-123: dense column-major P and extrinsic matrices (dim x dim+1),
//     the 100-entry LUT and the source-detector distance of the first pose.
// The matched (non-fast) Joseph adjoint, traverseAdjointKernel, is not exposed: the primary-axis
// voxel index of its atomic scatter is not clamped to the volume, so its bounds cannot be shown by
// reading and it is not run here.
// The 3D voxel kernel (traverseVolume3D) advances its detector pointer by nu + 1 - iStride after
// each footprint row (jStride, ProjectVoxelsCUDA.cu:147), where the CPU path advances by
// nu - iStride (VoxelComputation.h:88): row k of a footprint lands k pixels to the right, and on the last
// pose up to a footprint height past the sinogram's end. The harness therefore runs the voxel
// kernels on its own sinogram buffer padded by one pose (zeros), copying in and out.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "ProjectVoxelsCUDA.cuh"
#include "TraverseJosephsCUDA.cuh"
#include "TraverseSiddonsCUDA.cuh"

namespace
{
    constexpr int kLutSize = 100;   // Lut<float, DEFAULT_PROJECTOR_LUT_SIZE>, projectors/Luts.hpp:8
    constexpr int kPoseFloats = 40; // P 3x4 at 0, Pinv 4x3 at 12, C at 24, ext 3x4 at 27, sdd at 39
    thread_local std::string g_error;

    struct Fail {
        std::string msg;
    };

    void ck(cudaError_t e, const char* what)
    {
        if (e != cudaSuccess)
            throw Fail{std::string(what) + ": " + cudaGetErrorString(e)};
    }

    template <class F>
    int guard(F&& f)
    {
        try {
            f();
            return 0;
        } catch (const Fail& e) {
            g_error = e.msg;
        } catch (const std::exception& e) {
            g_error = e.what();
        }
        return 1;
    }
} // namespace

struct refcuda {
    unsigned nx = 0, ny = 0, nz = 0, nu = 0, nv = 0, np = 0;
    float sdd = 0.0f;
    // Joseph
    cudaPitchedPtr origins{}, projInv{}, proj{};
    cudaArray_t volArray = nullptr, sinoArray = nullptr;
    cudaTextureObject_t volTex = 0, sinoTex = 0;
    cudaPitchedPtr sinoPitched{}, volPitched{};
    // Siddon
    float* sidOrigins = nullptr;
    float* sidInv = nullptr;
    // voxel projectors
    float* voxProj = nullptr;
    float* voxExt = nullptr;
    float* lut = nullptr;
    float lutRadius = 0.0f;
    float* voxSino = nullptr; // (np + 1) poses: the last one absorbs the kernel's overrun

    ~refcuda()
    {
        if (volTex)
            cudaDestroyTextureObject(volTex);
        if (sinoTex)
            cudaDestroyTextureObject(sinoTex);
        if (volArray)
            cudaFreeArray(volArray);
        if (sinoArray)
            cudaFreeArray(sinoArray);
        for (void* p : {origins.ptr, projInv.ptr, proj.ptr, sinoPitched.ptr, volPitched.ptr,
                        static_cast<void*>(sidOrigins), static_cast<void*>(sidInv),
                        static_cast<void*>(voxProj), static_cast<void*>(voxExt),
                        static_cast<void*>(lut), static_cast<void*>(voxSino)})
            if (p)
                cudaFree(p);
    }

    size_t volBytes() const { return size_t(nx) * ny * nz * sizeof(float); }
    size_t sinoBytes() const { return size_t(nu) * nv * np * sizeof(float); }
};

namespace
{
    cudaTextureObject_t makeTexture(cudaArray_t array, bool border)
    {
        cudaResourceDesc res;
        std::memset(&res, 0, sizeof(res));
        res.resType = cudaResourceTypeArray;
        res.res.array.array = array;
        cudaTextureDesc tex;
        std::memset(&tex, 0, sizeof(tex));
        const auto mode = border ? cudaAddressModeBorder : cudaAddressModeClamp;
        tex.addressMode[0] = tex.addressMode[1] = tex.addressMode[2] = mode;
        tex.filterMode = cudaFilterModeLinear;
        tex.readMode = cudaReadModeElementType;
        tex.normalizedCoords = 0;
        cudaTextureObject_t t = 0;
        ck(cudaCreateTextureObject(&t, &res, &tex, nullptr), "cudaCreateTextureObject");
        return t;
    }

    // pitched (dim x dim per pose, column j of the block in pitched row j)
    void uploadBlocks(cudaPitchedPtr dst, const std::vector<float>& colMajor, unsigned np)
    {
        for (unsigned i = 0; i < np; ++i)
            ck(cudaMemcpy2D(static_cast<char*>(dst.ptr) + size_t(i) * dst.pitch * 3, dst.pitch,
                            colMajor.data() + 9 * size_t(i), 3 * sizeof(float), 3 * sizeof(float),
                            3, cudaMemcpyHostToDevice),
               "cudaMemcpy2D");
    }

    template <class T>
    T* deviceCopy(const std::vector<T>& h)
    {
        T* d = nullptr;
        ck(cudaMalloc(&d, h.size() * sizeof(T)), "cudaMalloc");
        ck(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
        return d;
    }
} // namespace

extern "C" {

const char* refcuda_last_error(void) { return g_error.c_str(); }

// 3D only: vol = (nx, ny, nz), det = (nu, nv, np), poses: np host pose records.
int refcuda_create(const int64_t* vol, const int64_t* det, const float* poses, refcuda** out)
{
    *out = nullptr;
    auto* h = new refcuda();
    const int rc = guard([&] {
        h->nx = unsigned(vol[0]), h->ny = unsigned(vol[1]), h->nz = unsigned(vol[2]);
        h->nu = unsigned(det[0]), h->nv = unsigned(det[1]), h->np = unsigned(det[2]);
        const unsigned np = h->np;
        h->sdd = poses[39];
        std::vector<float> inv(9 * size_t(np)), pblk(9 * size_t(np)), ro(3 * size_t(np)),
            centre(3 * size_t(np)), pFull(12 * size_t(np)), eFull(12 * size_t(np));
        for (unsigned i = 0; i < np; ++i) {
            const float* q = poses + size_t(i) * kPoseFloats;
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r) {
                    inv[9 * i + 3 * c + r] = q[12 + 3 * r + c]; // Pinv row r, column c
                    pblk[9 * i + 3 * c + r] = q[4 * r + c];     // P row r, column c
                }
            for (int c = 0; c < 4; ++c)
                for (int r = 0; r < 3; ++r) {
                    pFull[12 * i + 3 * c + r] = q[4 * r + c];
                    eFull[12 * i + 3 * c + r] = q[27 + 4 * r + c];
                }
            // ray origin = -Pinv_block * p4 (JosephsMethodCUDA.cpp:80-84)
            for (int r = 0; r < 3; ++r) {
                float s = 0.0f;
                for (int c = 0; c < 3; ++c)
                    s += q[12 + 3 * r + c] * q[4 * c + 3];
                ro[3 * i + r] = -s;
                centre[3 * i + r] = q[24 + r];
            }
        }
        // Joseph
        ck(cudaMallocPitch(&h->origins.ptr, &h->origins.pitch, 3 * sizeof(float), np),
           "cudaMallocPitch");
        ck(cudaMemcpy2D(h->origins.ptr, h->origins.pitch, ro.data(), 3 * sizeof(float),
                        3 * sizeof(float), np, cudaMemcpyHostToDevice),
           "cudaMemcpy2D");
        const cudaExtent mext = make_cudaExtent(3 * sizeof(float), 3, np);
        ck(cudaMalloc3D(&h->projInv, mext), "cudaMalloc3D");
        ck(cudaMalloc3D(&h->proj, mext), "cudaMalloc3D");
        uploadBlocks(h->projInv, inv, np);
        uploadBlocks(h->proj, pblk, np);
        const cudaChannelFormatDesc fd = cudaCreateChannelDesc(32, 0, 0, 0,
                                                               cudaChannelFormatKindFloat);
        ck(cudaMalloc3DArray(&h->volArray, &fd, make_cudaExtent(h->nx, h->ny, h->nz), 0),
           "cudaMalloc3DArray");
        h->volTex = makeTexture(h->volArray, false);
        ck(cudaMalloc3DArray(&h->sinoArray, &fd, make_cudaExtent(h->nu, h->nv, np),
                             cudaArrayLayered),
           "cudaMalloc3DArray");
        h->sinoTex = makeTexture(h->sinoArray, true);
        ck(cudaMalloc3D(&h->sinoPitched, make_cudaExtent(h->nu * sizeof(float), h->nv, np)),
           "cudaMalloc3D");
        ck(cudaMalloc3D(&h->volPitched, make_cudaExtent(h->nx * sizeof(float), h->ny, h->nz)),
           "cudaMalloc3D");
        // Siddon
        h->sidOrigins = deviceCopy(centre);
        h->sidInv = deviceCopy(inv);
        // voxel projectors
        h->voxProj = deviceCopy(pFull);
        h->voxExt = deviceCopy(eFull);
        ck(cudaMalloc(&h->voxSino, h->sinoBytes() + size_t(h->nu) * h->nv * sizeof(float)),
           "cudaMalloc");
    });
    if (rc) {
        delete h;
        return rc;
    }
    *out = h;
    return 0;
}

int refcuda_destroy(refcuda* h)
{
    delete h;
    return 0;
}

// ---- Joseph (texture forward, fast adjoint) -------------------------------------------------

// the per-call volume upload of JosephsMethodCUDA::copyTextureToGPU (device source here)
int refcuda_joseph_upload_volume(refcuda* h, const float* x)
{
    return guard([&] {
        cudaMemcpy3DParms p = {};
        p.srcPtr = make_cudaPitchedPtr(const_cast<float*>(x), h->nx * sizeof(float), h->nx, h->ny);
        p.dstArray = h->volArray;
        p.extent = make_cudaExtent(h->nx, h->ny, h->nz);
        p.kind = cudaMemcpyDeviceToDevice;
        ck(cudaMemcpy3DAsync(&p, 0), "cudaMemcpy3DAsync");
    });
}

int refcuda_joseph_forward(refcuda* h)
{
    return guard([&] {
        typename elsa::TraverseJosephsCUDA<float, 3>::BoundingBox box;
        box._max[0] = float(h->nx), box._max[1] = float(h->ny), box._max[2] = float(h->nz);
        const dim3 sinogramDims(h->np, h->nv, h->nu);
        elsa::TraverseJosephsCUDA<float, 3>::traverseForward(
            sinogramDims, elsa::TraverseJosephsCUDA<float, 3>::MAX_THREADS_PER_BLOCK, h->volTex,
            static_cast<int8_t*>(h->sinoPitched.ptr), h->sinoPitched.pitch,
            static_cast<int8_t*>(h->origins.ptr), uint32_t(h->origins.pitch),
            static_cast<int8_t*>(h->projInv.ptr), uint32_t(h->projInv.pitch), box);
        ck(cudaGetLastError(), "traverseForward");
    });
}

int refcuda_joseph_download_sinogram(refcuda* h, float* y)
{
    return guard([&] {
        ck(cudaMemcpy2DAsync(y, h->nu * sizeof(float), h->sinoPitched.ptr, h->sinoPitched.pitch,
                             h->nu * sizeof(float), size_t(h->nv) * h->np,
                             cudaMemcpyDeviceToDevice, 0),
           "cudaMemcpy2DAsync");
    });
}

// the per-call sinogram upload into the layered texture (copyTextureToGPU<cudaArrayLayered>)
int refcuda_joseph_upload_sinogram(refcuda* h, const float* y)
{
    return guard([&] {
        cudaMemcpy3DParms p = {};
        p.srcPtr = make_cudaPitchedPtr(const_cast<float*>(y), h->nu * sizeof(float), h->nu, h->nv);
        p.dstArray = h->sinoArray;
        p.extent = make_cudaExtent(h->nu, h->nv, h->np);
        p.kind = cudaMemcpyDeviceToDevice;
        ck(cudaMemcpy3DAsync(&p, 0), "cudaMemcpy3DAsync");
    });
}

int refcuda_joseph_adjoint_fast(refcuda* h)
{
    return guard([&] {
        const dim3 volumeDims(h->nz, h->ny, h->nx);
        elsa::TraverseJosephsCUDA<float, 3>::traverseAdjointFast(
            volumeDims, elsa::TraverseJosephsCUDA<float, 3>::MAX_THREADS_PER_BLOCK,
            static_cast<int8_t*>(h->volPitched.ptr), h->volPitched.pitch, h->sinoTex,
            static_cast<int8_t*>(h->origins.ptr), uint32_t(h->origins.pitch),
            static_cast<int8_t*>(h->proj.ptr), uint32_t(h->proj.pitch), h->np);
        ck(cudaGetLastError(), "traverseAdjointFast");
    });
}

int refcuda_joseph_download_volume(refcuda* h, float* x)
{
    return guard([&] {
        ck(cudaMemcpy2DAsync(x, h->nx * sizeof(float), h->volPitched.ptr, h->volPitched.pitch,
                             h->nx * sizeof(float), size_t(h->ny) * h->nz,
                             cudaMemcpyDeviceToDevice, 0),
           "cudaMemcpy2DAsync");
    });
}

// ---- Siddon ---------------------------------------------------------------------------------

int refcuda_siddon_forward(refcuda* h, const float* x, float* y)
{
    return guard([&] {
        ck(cudaMemsetAsync(y, 0, h->sinoBytes(), 0), "cudaMemsetAsync");
        typename elsa::TraverseSiddonsCUDA<float, 3>::BoundingBox box;
        box._max[0] = h->nx, box._max[1] = h->ny, box._max[2] = h->nz;
        const dim3 sinogramDims(h->np, h->nv, h->nu);
        elsa::TraverseSiddonsCUDA<float, 3>::traverseForward(
            sinogramDims, elsa::TraverseSiddonsCUDA<float, 3>::MAX_THREADS_PER_BLOCK,
            const_cast<float*>(x), h->nx, y, h->nu, h->sidOrigins, h->sidInv, box);
        ck(cudaGetLastError(), "Siddon traverseForward");
    });
}

int refcuda_siddon_adjoint(refcuda* h, const float* y, float* x)
{
    return guard([&] {
        ck(cudaMemsetAsync(x, 0, h->volBytes(), 0), "cudaMemsetAsync");
        typename elsa::TraverseSiddonsCUDA<float, 3>::BoundingBox box;
        box._max[0] = h->nx, box._max[1] = h->ny, box._max[2] = h->nz;
        const dim3 sinogramDims(h->np, h->nv, h->nu);
        elsa::TraverseSiddonsCUDA<float, 3>::traverseAdjoint(
            sinogramDims, elsa::TraverseSiddonsCUDA<float, 3>::MAX_THREADS_PER_BLOCK, x, h->nx,
            const_cast<float*>(y), h->nu, h->sidOrigins, h->sidInv, box);
        ck(cudaGetLastError(), "Siddon traverseAdjoint");
    });
}

// ---- blob / B-spline voxel projectors -------------------------------------------------------

// lut: 100 host floats on [0, radius] (Lut<float, 100>); radius = lut.support()
int refcuda_voxel_set_lut(refcuda* h, const float* lutHost, int32_t n, float radius)
{
    return guard([&] {
        if (n != kLutSize)
            throw Fail{"the reference kernels use a 100-entry LUT"};
        if (h->lut)
            cudaFree(h->lut);
        h->lut = deviceCopy(std::vector<float>(lutHost, lutHost + n));
        h->lutRadius = radius;
    });
}

// differential = 0: BlobVoxelProjectorCUDA / BSplineVoxelProjectorCUDA; 1: phase contrast
int refcuda_voxel_forward(refcuda* h, int32_t differential, const float* x, float* y)
{
    return guard([&] {
        if (!h->lut)
            throw Fail{"no LUT"};
        const size_t pad = size_t(h->nu) * h->nv * sizeof(float);
        ck(cudaMemsetAsync(h->voxSino, 0, h->sinoBytes() + pad, 0), "cudaMemsetAsync");
        ck(cudaStreamSynchronize(0), "cudaStreamSynchronize");
        const dim3 sinogramDims(h->nu, h->nv, h->np), volumeDims(h->nx, h->ny, h->nz);
        using namespace elsa;
        if (differential)
            ProjectVoxelsCUDA<float, 3, false, VoxelHelperCUDA::DIFFERENTIAL>::project(
                volumeDims, sinogramDims, ProjectVoxelsCUDA<float>::MAX_THREADS_PER_BLOCK,
                const_cast<float*>(x), h->voxSino, h->voxProj, h->voxExt, h->lut, h->lutRadius,
                h->sdd);
        else
            ProjectVoxelsCUDA<float, 3, false, VoxelHelperCUDA::CLASSIC>::project(
                volumeDims, sinogramDims, ProjectVoxelsCUDA<float>::MAX_THREADS_PER_BLOCK,
                const_cast<float*>(x), h->voxSino, h->voxProj, h->voxExt, h->lut, h->lutRadius,
                h->sdd);
        ck(cudaGetLastError(), "ProjectVoxelsCUDA forward");
        ck(cudaMemcpyAsync(y, h->voxSino, h->sinoBytes(), cudaMemcpyDeviceToDevice, 0),
           "cudaMemcpyAsync");
    });
}

int refcuda_voxel_adjoint(refcuda* h, int32_t differential, const float* y, float* x)
{
    return guard([&] {
        if (!h->lut)
            throw Fail{"no LUT"};
        const size_t pad = size_t(h->nu) * h->nv * sizeof(float);
        ck(cudaMemsetAsync(x, 0, h->volBytes(), 0), "cudaMemsetAsync");
        ck(cudaMemcpyAsync(h->voxSino, y, h->sinoBytes(), cudaMemcpyDeviceToDevice, 0),
           "cudaMemcpyAsync");
        ck(cudaMemsetAsync(reinterpret_cast<char*>(h->voxSino) + h->sinoBytes(), 0, pad, 0),
           "cudaMemsetAsync");
        ck(cudaStreamSynchronize(0), "cudaStreamSynchronize");
        const dim3 sinogramDims(h->nu, h->nv, h->np), volumeDims(h->nx, h->ny, h->nz);
        using namespace elsa;
        if (differential)
            ProjectVoxelsCUDA<float, 3, true, VoxelHelperCUDA::DIFFERENTIAL>::project(
                volumeDims, sinogramDims, ProjectVoxelsCUDA<float>::MAX_THREADS_PER_BLOCK, x,
                h->voxSino, h->voxProj, h->voxExt, h->lut, h->lutRadius, h->sdd);
        else
            ProjectVoxelsCUDA<float, 3, true, VoxelHelperCUDA::CLASSIC>::project(
                volumeDims, sinogramDims, ProjectVoxelsCUDA<float>::MAX_THREADS_PER_BLOCK, x,
                h->voxSino, h->voxProj, h->voxExt, h->lut, h->lutRadius, h->sdd);
        ck(cudaGetLastError(), "ProjectVoxelsCUDA adjoint");
    });
}

// ---- 2D Joseph fast adjoint (JosephsMethodCUDA.cpp:300-335) ------------------------------------

struct refcuda2d {
    unsigned nx = 0, ny = 0, nu = 0, np = 0;
    cudaPitchedPtr origins{}, proj{}, volPitched{};
    cudaArray_t sinoArray = nullptr;
    cudaTextureObject_t sinoTex = 0;
    ~refcuda2d()
    {
        if (sinoTex)
            cudaDestroyTextureObject(sinoTex);
        if (sinoArray)
            cudaFreeArray(sinoArray);
        for (void* p : {origins.ptr, proj.ptr, volPitched.ptr})
            if (p)
                cudaFree(p);
    }
};

// vol = (nx, ny), det = (nu, np), poses: np host 2D pose records (P 2x3 at 0, Pinv 3x2 at 12)
int refcuda2d_create(const int64_t* vol, const int64_t* det, const float* poses, refcuda2d** out)
{
    *out = nullptr;
    auto* h = new refcuda2d();
    const int rc = guard([&] {
        h->nx = unsigned(vol[0]), h->ny = unsigned(vol[1]);
        h->nu = unsigned(det[0]), h->np = unsigned(det[1]);
        const unsigned np = h->np;
        std::vector<float> pblk(4 * size_t(np)), ro(2 * size_t(np));
        for (unsigned i = 0; i < np; ++i) {
            const float* q = poses + size_t(i) * kPoseFloats;
            for (int c = 0; c < 2; ++c)
                for (int r = 0; r < 2; ++r)
                    pblk[4 * i + 2 * c + r] = q[3 * r + c];
            for (int r = 0; r < 2; ++r) {
                float s = 0.0f;
                for (int c = 0; c < 2; ++c)
                    s += q[12 + 2 * r + c] * q[3 * c + 2];
                ro[2 * i + r] = -s;
            }
        }
        ck(cudaMallocPitch(&h->origins.ptr, &h->origins.pitch, 2 * sizeof(float), np),
           "cudaMallocPitch");
        ck(cudaMemcpy2D(h->origins.ptr, h->origins.pitch, ro.data(), 2 * sizeof(float),
                        2 * sizeof(float), np, cudaMemcpyHostToDevice),
           "cudaMemcpy2D");
        ck(cudaMalloc3D(&h->proj, make_cudaExtent(2 * sizeof(float), 2, np)), "cudaMalloc3D");
        for (unsigned i = 0; i < np; ++i)
            ck(cudaMemcpy2D(static_cast<char*>(h->proj.ptr) + size_t(i) * h->proj.pitch * 2,
                            h->proj.pitch, pblk.data() + 4 * size_t(i), 2 * sizeof(float),
                            2 * sizeof(float), 2, cudaMemcpyHostToDevice),
               "cudaMemcpy2D");
        const cudaChannelFormatDesc fd = cudaCreateChannelDesc(32, 0, 0, 0,
                                                               cudaChannelFormatKindFloat);
        // a layered 1D array is a 3D array of height 0 (JosephsMethodCUDA.cpp:504-512)
        ck(cudaMalloc3DArray(&h->sinoArray, &fd, make_cudaExtent(h->nu, 0, np), cudaArrayLayered),
           "cudaMalloc3DArray");
        h->sinoTex = makeTexture(h->sinoArray, true);
        ck(cudaMallocPitch(&h->volPitched.ptr, &h->volPitched.pitch, h->nx * sizeof(float),
                           h->ny),
           "cudaMallocPitch");
    });
    if (rc) {
        delete h;
        return rc;
    }
    *out = h;
    return 0;
}

int refcuda2d_destroy(refcuda2d* h)
{
    delete h;
    return 0;
}

// y (device, nu * np) -> x (device, nx * ny): sinogram upload, fast adjoint kernel, copy out
int refcuda2d_joseph_adjoint_fast(refcuda2d* h, const float* y, float* x)
{
    return guard([&] {
        cudaMemcpy3DParms p = {};
        p.srcPtr = make_cudaPitchedPtr(const_cast<float*>(y), h->nu * sizeof(float), h->nu, 1);
        p.dstArray = h->sinoArray;
        p.extent = make_cudaExtent(h->nu, 1, h->np);
        p.kind = cudaMemcpyDeviceToDevice;
        ck(cudaMemcpy3DAsync(&p, 0), "cudaMemcpy3DAsync");
        const dim3 volumeDims(1, h->ny, h->nx);
        elsa::TraverseJosephsCUDA<float, 2>::traverseAdjointFast(
            volumeDims, elsa::TraverseJosephsCUDA<float, 2>::MAX_THREADS_PER_BLOCK,
            static_cast<int8_t*>(h->volPitched.ptr), h->volPitched.pitch, h->sinoTex,
            static_cast<int8_t*>(h->origins.ptr), uint32_t(h->origins.pitch),
            static_cast<int8_t*>(h->proj.ptr), uint32_t(h->proj.pitch), h->np);
        ck(cudaGetLastError(), "traverseAdjointFast 2D");
        ck(cudaMemcpy2DAsync(x, h->nx * sizeof(float), h->volPitched.ptr, h->volPitched.pitch,
                             h->nx * sizeof(float), h->ny, cudaMemcpyDeviceToDevice, 0),
           "cudaMemcpy2DAsync");
    });
}

} // extern "C"
