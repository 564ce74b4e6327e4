// C ABI of elsa_b200 (include/elsa_b200.h): argument checks, exception -> status translation.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/elsa_b200.h"
#include "geometry.hpp"
#include "internal.cuh"
#include "io.hpp"
#include "projector.hpp"
#include "solvers.hpp"
#include "tune.hpp"
#include "voxel.hpp"

struct elsa_solver {
    std::unique_ptr<elsa_b200::SolverSession> impl;
    int device = 0;
};

struct elsa_batch_cgne {
    std::unique_ptr<elsa_b200::BatchedCgne> impl;
    int device = 0;
};

struct elsa_cgne_split {
    std::unique_ptr<elsa_b200::SplitCgne> impl;
    int device = 0;
};

struct elsa_projector {
    std::unique_ptr<elsa_b200::Projector> impl;
    // lazily allocated staging buffers of the host-buffer entry points
    std::unique_ptr<elsa_b200::DeviceBuffer> hostIn, hostOut;
    // streams (compute, copy) and per-group events of the pipelined host-buffer entry points;
    // blocking streams, so they order with the legacy default stream as a synchronous copy does
    cudaStream_t hostCompute = nullptr, hostCopy = nullptr;
    std::vector<cudaEvent_t> hostEvents;
    ~elsa_projector()
    {
        // streams and events belong to the projector's device: destroy them with it current
        int prev = -1;
        const bool any = hostCompute || hostCopy || !hostEvents.empty();
        if (any && impl && cudaGetDevice(&prev) == cudaSuccess && prev != impl->device())
            cudaSetDevice(impl->device());
        else
            prev = -1;
        for (cudaEvent_t e : hostEvents)
            cudaEventDestroy(e);
        if (hostCompute)
            cudaStreamDestroy(hostCompute);
        if (hostCopy)
            cudaStreamDestroy(hostCopy);
        if (prev >= 0)
            cudaSetDevice(prev);
    }
};

namespace
{
    thread_local std::string gLastError;

    template <class Fn>
    elsa_status guarded(Fn&& fn)
    {
        try {
            fn();
            gLastError.clear();
            return ELSA_SUCCESS;
        } catch (const elsa_b200::Error& e) {
            gLastError = e.what();
            return e.status;
        } catch (const std::bad_alloc& e) {
            gLastError = e.what();
            return ELSA_ERROR_BAD_ALLOC;
        } catch (const std::exception& e) {
            gLastError = e.what();
            return ELSA_ERROR_LOGIC;
        } catch (...) {
            gLastError = "unknown error";
            return ELSA_ERROR_LOGIC;
        }
    }

    void require(bool cond, const char* msg)
    {
        if (!cond)
            throw elsa_b200::Error(ELSA_ERROR_INVALID_ARGUMENT, msg);
    }

    cudaStream_t asStream(void* s)
    {
        return static_cast<cudaStream_t>(s);
    }

    void onDevice(const elsa_projector* p)
    {
        int cur = 0;
        ELSA_CUDA(cudaGetDevice(&cur));
        if (cur != p->impl->device())
            ELSA_CUDA(cudaSetDevice(p->impl->device()));
    }
} // namespace

namespace
{
    struct VoxelSpec {
        elsa_b200::VoxelLut lut;
        bool phase = false;
        elsa_b200::FootprintMode mode = elsa_b200::FootprintMode::Reference;
    };

    // Parameters of the voxel projector kinds (elsa_b200.h): blob (radius, alpha, order, mode),
    // B-spline (order, mode); the lookup table of the absorption or phase-contrast variant.
    VoxelSpec voxelSpec(int32_t kind, int32_t dim, const float* params, int32_t numParams)
    {
        const bool blob = kind == ELSA_PROJECTOR_BLOB || kind == ELSA_PROJECTOR_PHASE_CONTRAST_BLOB;
        const bool phase = kind == ELSA_PROJECTOR_PHASE_CONTRAST_BLOB ||
                           kind == ELSA_PROJECTOR_PHASE_CONTRAST_BSPLINE;
        if (!blob && kind != ELSA_PROJECTOR_BSPLINE && !phase)
            throw elsa_b200::Error(ELSA_ERROR_NOT_SUPPORTED, "not a voxel projector kind");
        if (dim != 2 && dim != 3)
            throw elsa_b200::Error(ELSA_ERROR_INVALID_ARGUMENT,
                                   "voxel projector: only supporting 2d/3d operations");
        const int maxParams = blob ? 4 : 2;
        if (numParams > maxParams)
            throw elsa_b200::Error(ELSA_ERROR_INVALID_ARGUMENT,
                                   "voxel projector: too many parameters");
        auto param = [&](int i, float dflt) { return i < numParams ? params[i] : dflt; };
        auto asInt = [](float v, const char* what) {
            if (!(v == std::floor(v)) || v < 0.0f || v > 64.0f)
                throw elsa_b200::Error(ELSA_ERROR_INVALID_ARGUMENT,
                                       std::string("voxel projector: invalid ") + what);
            return static_cast<int>(v);
        };
        const auto profile = !phase ? elsa_b200::LutProfile::Value
                                    : (dim == 2 ? elsa_b200::LutProfile::Derivative
                                                : elsa_b200::LutProfile::NormalizedGradient);
        VoxelSpec spec;
        spec.phase = phase;
        int mode;
        if (blob) {
            const float radius = param(0, 2.0f);
            const float alpha = param(1, 10.83f);
            const int order = asInt(param(2, 2.0f), "blob order");
            if (phase && order < 1)
                throw elsa_b200::Error(ELSA_ERROR_INVALID_ARGUMENT,
                                       "phase-contrast blob: order must be 1 or 2");
            spec.lut = elsa_b200::blobLut(radius, alpha, order, profile);
            mode = asInt(param(3, 0.0f), "footprint mode");
        } else {
            const int order = asInt(param(0, 2.0f), "B-spline order");
            spec.lut = elsa_b200::bsplineLut(dim, order, profile);
            mode = asInt(param(1, 0.0f), "footprint mode");
        }
        if (mode > 1)
            throw elsa_b200::Error(ELSA_ERROR_INVALID_ARGUMENT,
                                   "voxel projector: footprint mode must be 0 or 1");
        spec.mode = static_cast<elsa_b200::FootprintMode>(mode);
        return spec;
    }
} // namespace

extern "C" {

const char* elsa_last_error(void)
{
    return gLastError.c_str();
}

int32_t elsa_abi_version(void)
{
    return 1;
}

elsa_status elsa_pose_2d(float s2c, float c2d, float angle, const float* volSpacing,
                         const float* volOrigin, const float* sinoSpacing, const float* sinoOrigin,
                         float ppOffset, const float* corOffset, float* out)
{
    return guarded([&] {
        require(volSpacing && volOrigin && sinoSpacing && sinoOrigin && corOffset && out,
                "elsa_pose_2d: null argument");
        const auto rec = elsa_b200::makePose2d(s2c, c2d, angle, volSpacing, volOrigin,
                                               sinoSpacing, sinoOrigin, ppOffset, corOffset);
        std::memcpy(out, rec.v, sizeof(rec.v));
    });
}

elsa_status elsa_pose_3d(float s2c, float c2d, const float* volSpacing, const float* volOrigin,
                         const float* sinoSpacing, const float* sinoOrigin, float gamma,
                         float beta, float alpha, const float* ppOffset, const float* corOffset,
                         float* out)
{
    return guarded([&] {
        require(volSpacing && volOrigin && sinoSpacing && sinoOrigin && ppOffset && corOffset &&
                    out,
                "elsa_pose_3d: null argument");
        const auto rec = elsa_b200::makePose3d(s2c, c2d, volSpacing, volOrigin, sinoSpacing,
                                               sinoOrigin, gamma, beta, alpha, ppOffset,
                                               corOffset);
        std::memcpy(out, rec.v, sizeof(rec.v));
    });
}

elsa_status elsa_circle_trajectory(int32_t dim, const int64_t* volDims, const float* volSpacing,
                                   int64_t numPoses, float arc, float s2c, float c2d,
                                   const int64_t* detSize, const float* detSpacing,
                                   float* outPoses, int64_t* outDetDims)
{
    return guarded([&] {
        require(dim == 2 || dim == 3, "CircleTrajectoryGenerator: can only handle 2d/3d");
        require(volDims && volSpacing && outPoses && outDetDims,
                "elsa_circle_trajectory: null argument");
        require(numPoses > 0, "elsa_circle_trajectory: need at least one pose");
        const auto poses = elsa_b200::circleTrajectory(dim, volDims, volSpacing, numPoses, arc,
                                                       s2c, c2d, detSize, detSpacing, outDetDims);
        std::memcpy(outPoses, poses.data(), sizeof(elsa_b200::PoseRecord) * poses.size());
    });
}

static elsa_status projectorCreate(int32_t kind, int32_t dim, const int64_t* volDims,
                                   const int64_t* detDims, const float* poses, const float* params,
                                   int32_t numParams, const elsa_b200::CurvedDetector& curved,
                                   elsa_projector** out)
{
    return guarded([&] {
        require(out != nullptr, "elsa_projector_create: null output handle");
        *out = nullptr;
        require(dim == 2 || dim == 3, "JosephsMethod: only supporting 2d/3d operations");
        require(volDims && detDims && poses, "elsa_projector_create: null argument");
        require(numParams >= 0 && (numParams == 0 || params != nullptr),
                "elsa_projector_create: invalid parameter array");
        for (int i = 0; i < dim; ++i) {
            require(volDims[i] > 0 && volDims[i] < (1 << 20),
                    "elsa_projector_create: invalid volume size");
            require(detDims[i] > 0 && detDims[i] < (1 << 24),
                    "elsa_projector_create: invalid detector size");
        }
        require(detDims[dim - 1] > 0, "JosephsMethod: geometry list was empty");
        elsa_b200::VolumeShape vol{dim, {static_cast<int>(volDims[0]),
                                         static_cast<int>(volDims[1]),
                                         dim == 3 ? static_cast<int>(volDims[2]) : 1}};
        elsa_b200::DetectorShape det{static_cast<int>(detDims[0]),
                                     dim == 3 ? static_cast<int>(detDims[1]) : 1,
                                     static_cast<int>(detDims[dim - 1])};
        std::vector<elsa_b200::PoseRecord> pv(static_cast<size_t>(det.np));
        std::memcpy(pv.data(), poses, sizeof(elsa_b200::PoseRecord) * pv.size());
        auto handle = std::make_unique<elsa_projector>();
        switch (kind) {
        case ELSA_PROJECTOR_JOSEPH: {
            require(numParams <= 1, "JosephsMethod: too many parameters");
            const bool fast = numParams >= 1 && params[0] != 0.0f;
            if (fast && curved.enabled())
                throw elsa_b200::Error(ELSA_ERROR_NOT_SUPPORTED,
                                       "JosephsMethodCUDA: the fast adjoint needs a planar "
                                       "detector");
            handle->impl = elsa_b200::makeJosephProjector(vol, det, pv, curved, fast);
            break;
        }
        case ELSA_PROJECTOR_SIDDON:
            handle->impl = elsa_b200::makeSiddonProjector(vol, det, pv, false, curved);
            break;
        case ELSA_PROJECTOR_BINARY:
            handle->impl = elsa_b200::makeSiddonProjector(vol, det, pv, true, curved);
            break;
        case ELSA_PROJECTOR_RAY_BLOB:
        case ELSA_PROJECTOR_RAY_BSPLINE: {
            if (curved.enabled())
                throw elsa_b200::Error(ELSA_ERROR_NOT_SUPPORTED,
                                       "LutProjector: curved detectors are not supported");
            const bool blob = kind == ELSA_PROJECTOR_RAY_BLOB;
            require(numParams <= (blob ? 3 : 1), "LutProjector: too many parameters");
            const VoxelSpec spec = voxelSpec(blob ? ELSA_PROJECTOR_BLOB : ELSA_PROJECTOR_BSPLINE,
                                             dim, params, numParams);
            // BlobProjector::support = ceil(radius), BSplineProjector::support = 2
            // (projectors/LutProjector.h:199, LutProjector.cpp:77-80)
            const int support = blob ? static_cast<int>(std::ceil(spec.lut.support)) : 2;
            handle->impl = elsa_b200::makeLutProjector(kind, vol, det, pv, spec.lut, support);
            break;
        }
        case ELSA_PROJECTOR_BLOB:
        case ELSA_PROJECTOR_BSPLINE:
        case ELSA_PROJECTOR_PHASE_CONTRAST_BLOB:
        case ELSA_PROJECTOR_PHASE_CONTRAST_BSPLINE: {
            if (curved.enabled())
                throw elsa_b200::Error(ELSA_ERROR_NOT_SUPPORTED,
                                       "voxel projectors need a planar detector");
            const VoxelSpec spec = voxelSpec(kind, dim, params, numParams);
            handle->impl = elsa_b200::makeVoxelProjector(kind, vol, det, pv, spec.lut,
                                                         spec.phase, spec.mode);
            break;
        }
        default:
            throw elsa_b200::Error(ELSA_ERROR_NOT_SUPPORTED, "unknown projector kind");
        }
        *out = handle.release();
    });
}

elsa_status elsa_projector_create(int32_t kind, int32_t dim, const int64_t* volDims,
                                  const int64_t* detDims, const float* poses, const float* params,
                                  int32_t numParams, elsa_projector** out)
{
    return projectorCreate(kind, dim, volDims, detDims, poses, params, numParams, {}, out);
}

elsa_status elsa_projector_create_curved(int32_t kind, int32_t dim, const int64_t* volDims,
                                         const int64_t* detDims, const float* poses,
                                         const float* params, int32_t numParams, float angle,
                                         float s2d, elsa_projector** out)
{
    if (!(angle > 0.0f) || !(s2d > 0.0f)) {
        gLastError = "CurvedDetectorDescriptor: angle and source-to-detector distance must be "
                     "positive";
        if (out)
            *out = nullptr;
        return ELSA_ERROR_INVALID_ARGUMENT;
    }
    elsa_b200::CurvedDetector c;
    c.angle = angle;
    c.s2d = s2d;
    return projectorCreate(kind, dim, volDims, detDims, poses, params, numParams, c, out);
}

elsa_status elsa_curved_detector_coords(int32_t dim, int32_t nu, int32_t nv, float angle,
                                        float s2d, float* out)
{
    return guarded([&] {
        require(out != nullptr, "elsa_curved_detector_coords: null output");
        require(dim == 2 || dim == 3, "elsa_curved_detector_coords: dim must be 2 or 3");
        require(nu > 0 && (dim == 2 || nv > 0), "elsa_curved_detector_coords: empty detector");
        require(angle > 0.0f && s2d > 0.0f,
                "CurvedDetectorDescriptor: angle and source-to-detector distance must be "
                "positive");
        const std::vector<float> xy =
            elsa_b200::curvedPlanarCoords(dim, nu, dim == 3 ? nv : 1, angle, s2d);
        std::memcpy(out, xy.data(), sizeof(float) * xy.size());
    });
}

elsa_status elsa_voxel_lut(int32_t kind, int32_t dim, const float* params, int32_t numParams,
                           int32_t samples, float* out, float* support)
{
    return guarded([&] {
        require(out && support && samples >= 2 && samples <= 1 << 20,
                "elsa_voxel_lut: invalid argument");
        require(numParams >= 0 && (numParams == 0 || params != nullptr),
                "elsa_voxel_lut: invalid parameter array");
        VoxelSpec spec = voxelSpec(kind, dim, params, numParams);
        if (samples != elsa_b200::kVoxelLutSize) {
            // same profile with another sample count (the reference's Lut<data_t, N>)
            const bool blob =
                kind == ELSA_PROJECTOR_BLOB || kind == ELSA_PROJECTOR_PHASE_CONTRAST_BLOB;
            const auto profile = !spec.phase ? elsa_b200::LutProfile::Value
                                             : (dim == 2 ? elsa_b200::LutProfile::Derivative
                                                         : elsa_b200::LutProfile::NormalizedGradient);
            auto p = [&](int i, float d) { return i < numParams ? params[i] : d; };
            spec.lut = blob ? elsa_b200::blobLut(p(0, 2.0f), p(1, 10.83f),
                                                 static_cast<int>(p(2, 2.0f)), profile, samples)
                            : elsa_b200::bsplineLut(dim, static_cast<int>(p(0, 2.0f)), profile,
                                                    samples);
        }
        std::memcpy(out, spec.lut.values.data(), sizeof(float) * spec.lut.values.size());
        *support = spec.lut.support;
    });
}

elsa_status elsa_projector_destroy(elsa_projector* p)
{
    return guarded([&] { delete p; });
}

elsa_status elsa_projector_sizes(const elsa_projector* p, int64_t* domain, int64_t* range)
{
    return guarded([&] {
        require(p && domain && range, "elsa_projector_sizes: null argument");
        *domain = p->impl->domainSize();
        *range = p->impl->rangeSize();
    });
}

elsa_status elsa_projector_info(const elsa_projector* p, int32_t key, int64_t* value)
{
    return guarded([&] {
        require(p && value, "elsa_projector_info: null argument");
        *value = p->impl->info(key);
    });
}

elsa_status elsa_projector_wait_test(elsa_projector* p, int64_t waitCycles, int32_t withholdCopies)
{
    return guarded([&] {
        require(p, "elsa_projector_wait_test: null argument");
        onDevice(p);
        if (!p->impl->setWaitTest(waitCycles, withholdCopies != 0))
            throw elsa_b200::Error(ELSA_ERROR_NOT_SUPPORTED,
                                   "elsa_projector_wait_test: this projector has no bounded "
                                   "device waits");
    });
}

elsa_status elsa_projector_get_knob(const elsa_projector* p, int32_t knob, int32_t* value)
{
    return guarded([&] {
        require(p && value, "elsa_projector_get_knob: null argument");
        require(knob >= 0 && knob < ELSA_KNOB_COUNT, "elsa_projector_get_knob: unknown knob");
        *value = p->impl->knob(knob);
    });
}

elsa_status elsa_projector_knob_candidates(const elsa_projector* p, int32_t knob,
                                           int32_t* values, int32_t capacity, int32_t* count)
{
    return guarded([&] {
        require(p && count, "elsa_projector_knob_candidates: null argument");
        require(knob >= 0 && knob < ELSA_KNOB_COUNT,
                "elsa_projector_knob_candidates: unknown knob");
        require(capacity >= 0 && (capacity == 0 || values),
                "elsa_projector_knob_candidates: bad output buffer");
        const std::vector<int> c = p->impl->knobCandidates(knob);
        *count = static_cast<int32_t>(c.size());
        for (int32_t i = 0; i < capacity && i < static_cast<int32_t>(c.size()); ++i)
            values[i] = c[i];
    });
}

elsa_status elsa_projector_set_knob(elsa_projector* p, int32_t knob, int32_t value)
{
    return guarded([&] {
        require(p, "elsa_projector_set_knob: null argument");
        require(knob >= 0 && knob < ELSA_KNOB_COUNT, "elsa_projector_set_knob: unknown knob");
        onDevice(p);
        ELSA_CUDA(cudaDeviceSynchronize()); // no launch of the old configuration in flight
        p->impl->setKnob(knob, value);
    });
}

elsa_status elsa_projector_autotune(elsa_projector* p, void* stream, int32_t force,
                                    int32_t* values, int32_t* fromCache)
{
    return guarded([&] {
        require(p, "elsa_projector_autotune: null argument");
        onDevice(p);
        ELSA_CUDA(cudaStreamSynchronize(asStream(stream)));
        const elsa_b200::TuneResult r =
            elsa_b200::autotune(*p->impl, asStream(stream), force != 0);
        if (values)
            for (int k = 0; k < ELSA_KNOB_COUNT; ++k)
                values[k] = r.values[k];
        if (fromCache)
            *fromCache = r.fromCache ? 1 : 0;
    });
}

elsa_status elsa_tune_cache_size(int64_t* entries)
{
    return guarded([&] {
        require(entries != nullptr, "elsa_tune_cache_size: null argument");
        *entries = static_cast<int64_t>(elsa_b200::tuneCacheSize());
    });
}

elsa_status elsa_tune_cache_clear(void)
{
    return guarded([&] { elsa_b200::tuneCacheClear(); });
}

elsa_status elsa_tune_cache_save(const char* path)
{
    return guarded([&] {
        require(path != nullptr, "elsa_tune_cache_save: null path");
        elsa_b200::tuneCacheSave(path);
    });
}

elsa_status elsa_tune_cache_load(const char* path)
{
    return guarded([&] {
        require(path != nullptr, "elsa_tune_cache_load: null path");
        elsa_b200::tuneCacheLoad(path);
    });
}

elsa_status elsa_tune_cache_put(const char* key, const int32_t* values)
{
    return guarded([&] {
        require(key && values, "elsa_tune_cache_put: null argument");
        elsa_b200::KnobValues v{};
        for (int k = 0; k < ELSA_KNOB_COUNT; ++k) {
            require(values[k] >= -1, "elsa_tune_cache_put: knob values must be >= -1");
            v[k] = values[k];
        }
        elsa_b200::tuneCachePut(key, v);
    });
}

elsa_status elsa_tune_cache_get(const char* key, int32_t* values, int32_t* found)
{
    return guarded([&] {
        require(key && values && found, "elsa_tune_cache_get: null argument");
        elsa_b200::KnobValues v{};
        const bool hit = elsa_b200::tuneCacheGet(key, v);
        *found = hit ? 1 : 0;
        if (hit)
            for (int k = 0; k < ELSA_KNOB_COUNT; ++k)
                values[k] = v[k];
    });
}

elsa_status elsa_projector_apply(elsa_projector* p, const float* x, float* y, void* stream)
{
    return guarded([&] {
        require(p && x && y, "elsa_projector_apply: null argument");
        onDevice(p);
        p->impl->forward(x, y, asStream(stream));
    });
}

elsa_status elsa_projector_apply_adjoint(elsa_projector* p, const float* y, float* x,
                                         void* stream)
{
    return guarded([&] {
        require(p && x && y, "elsa_projector_apply_adjoint: null argument");
        onDevice(p);
        p->impl->adjoint(y, x, asStream(stream));
    });
}

elsa_status elsa_projector_apply_batch(elsa_projector* p, const float* x, int64_t xStride,
                                       float* y, int64_t yStride, int32_t batch, void* stream)
{
    return guarded([&] {
        require(p && batch >= 0 && (batch == 0 || (x && y)),
                "elsa_projector_apply_batch: invalid argument");
        require(batch <= 1 || (xStride >= p->impl->domainSize() && yStride >= p->impl->rangeSize()),
                "elsa_projector_apply_batch: strides must not make the elements overlap");
        onDevice(p);
        p->impl->forwardBatch(x, xStride, y, yStride, batch, asStream(stream));
    });
}

elsa_status elsa_projector_apply_adjoint_batch(elsa_projector* p, const float* y, int64_t yStride,
                                               float* x, int64_t xStride, int32_t batch,
                                               void* stream)
{
    return guarded([&] {
        require(p && batch >= 0 && (batch == 0 || (x && y)),
                "elsa_projector_apply_adjoint_batch: invalid argument");
        require(batch <= 1 || (xStride >= p->impl->domainSize() && yStride >= p->impl->rangeSize()),
                "elsa_projector_apply_adjoint_batch: strides must not make the elements overlap");
        onDevice(p);
        p->impl->adjointBatch(y, yStride, x, xStride, batch, asStream(stream));
    });
}

static void hostApply(elsa_projector* p, const float* in, float* out, bool adjoint)
{
    onDevice(p);
    const int64_t nin = adjoint ? p->impl->rangeSize() : p->impl->domainSize();
    const int64_t nout = adjoint ? p->impl->domainSize() : p->impl->rangeSize();
    const size_t need = sizeof(float) * static_cast<size_t>(std::max(nin, nout));
    if (!p->hostIn || p->hostIn->bytes() < need) {
        p->hostIn = std::make_unique<elsa_b200::DeviceBuffer>(need);
        p->hostOut = std::make_unique<elsa_b200::DeviceBuffer>(need);
    }
    float* din = p->hostIn->as<float>();
    float* dout = p->hostOut->as<float>();
    elsa_b200::Projector& P = *p->impl;
    const int groups = adjoint ? P.adjointGroups() : P.forwardGroups();
    if (groups > 1) {
        // Pipelined: the forward's finished view groups are copied out while later groups run;
        // the adjoint's view groups are copied in while earlier groups run.
        if (!p->hostCompute) {
            ELSA_CUDA(cudaStreamCreate(&p->hostCompute));
            ELSA_CUDA(cudaStreamCreate(&p->hostCopy));
        }
        while (static_cast<int>(p->hostEvents.size()) < groups) {
            cudaEvent_t e = nullptr;
            ELSA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            p->hostEvents.push_back(e);
        }
        cudaStream_t sc = p->hostCompute, sx = p->hostCopy;
        const int64_t view = P.rangeSize() / P.detector().np;
        try {
        if (!adjoint) {
            ELSA_CUDA(cudaMemcpyAsync(din, in, sizeof(float) * nin, cudaMemcpyHostToDevice, sc));
            P.prepareForward(din, sc);
            for (int g = 0; g < groups; ++g) {
                P.forwardGroup(din, dout, g, groups, sc);
                ELSA_CUDA(cudaEventRecord(p->hostEvents[g], sc));
                ELSA_CUDA(cudaStreamWaitEvent(sx, p->hostEvents[g], 0));
                const auto v = P.forwardGroupViews(g, groups);
                ELSA_CUDA(cudaMemcpyAsync(out + v.first * view, dout + v.first * view,
                                          sizeof(float) * (v.second - v.first) * view,
                                          cudaMemcpyDeviceToHost, sx));
            }
            ELSA_CUDA(cudaStreamSynchronize(sx));
        } else {
            for (int g = 0; g < groups; ++g) {
                const auto v = P.adjointGroupViews(g, groups);
                ELSA_CUDA(cudaMemcpyAsync(din + v.first * view, in + v.first * view,
                                          sizeof(float) * (v.second - v.first) * view,
                                          cudaMemcpyHostToDevice, sx));
                ELSA_CUDA(cudaEventRecord(p->hostEvents[g], sx));
                ELSA_CUDA(cudaStreamWaitEvent(sc, p->hostEvents[g], 0));
                P.adjointGroup(din, g, groups, sc);
            }
            P.adjointFinish(dout, sc);
            ELSA_CUDA(cudaMemcpyAsync(out, dout, sizeof(float) * nout, cudaMemcpyDeviceToHost,
                                      sc));
            ELSA_CUDA(cudaStreamSynchronize(sc));
        }
        } catch (...) {
            // copies into or out of the caller's buffers may still be queued: finish them
            // before the error returns, so that no late copy touches a buffer the caller reuses
            cudaStreamSynchronize(sc);
            cudaStreamSynchronize(sx);
            throw;
        }
        return;
    }
    ELSA_CUDA(cudaMemcpy(din, in, sizeof(float) * nin, cudaMemcpyHostToDevice));
    if (adjoint)
        p->impl->adjoint(din, dout, nullptr);
    else
        p->impl->forward(din, dout, nullptr);
    ELSA_CUDA(cudaMemcpy(out, dout, sizeof(float) * nout, cudaMemcpyDeviceToHost));
}

elsa_status elsa_projector_apply_host(elsa_projector* p, const float* x, float* y)
{
    return guarded([&] {
        require(p && x && y, "elsa_projector_apply_host: null argument");
        hostApply(p, x, y, false);
    });
}

elsa_status elsa_projector_apply_adjoint_host(elsa_projector* p, const float* y, float* x)
{
    return guarded([&] {
        require(p && x && y, "elsa_projector_apply_adjoint_host: null argument");
        hostApply(p, y, x, true);
    });
}

namespace
{
    // The partial sums of one reduction, taken from the device's stream-ordered memory pool on
    // the call's stream and returned to it on the same stream: no device-wide synchronization
    // (as cudaMalloc/cudaFree have), no wait on the host, and calls on different streams get
    // separate buffers.
    class StreamPartials
    {
    public:
        explicit StreamPartials(cudaStream_t s) : s_(s)
        {
            ELSA_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p_),
                                      sizeof(double) * elsa_b200::kReduceBlocks, s_));
        }
        ~StreamPartials() { cudaFreeAsync(p_, s_); }
        StreamPartials(const StreamPartials&) = delete;
        StreamPartials& operator=(const StreamPartials&) = delete;
        double* get() const { return p_; }

    private:
        cudaStream_t s_;
        double* p_ = nullptr;
    };
} // namespace

elsa_status elsa_dot(const float* x, const float* y, int64_t n, double* result, void* stream)
{
    return guarded([&] {
        require(result && n >= 0 && ((x && y) || n == 0), "elsa_dot: invalid argument");
        StreamPartials partials(asStream(stream));
        elsa_b200::launchDot(x, y, n, partials.get(), result, asStream(stream));
    });
}

elsa_status elsa_dot_no_alloc(const float* x, const float* y, int64_t n, double* result,
                              void* stream)
{
    return guarded([&] { elsa_b200::dotNoAlloc(x, y, n, result, asStream(stream)); });
}

elsa_status elsa_squared_l2_norm(const float* x, int64_t n, double* result, void* stream)
{
    return guarded([&] {
        require(result && n >= 0 && (x || n == 0), "elsa_squared_l2_norm: invalid argument");
        StreamPartials partials(asStream(stream));
        elsa_b200::launchSquaredNorm(x, n, partials.get(), result, asStream(stream));
    });
}

elsa_status elsa_lincomb(float a, const float* x, float b, const float* y, float* out, int64_t n,
                         void* stream)
{
    return guarded([&] {
        require(n >= 0 && ((x && y && out) || n == 0), "elsa_lincomb: invalid argument");
        elsa_b200::launchLincomb(a, x, b, y, out, n, asStream(stream));
    });
}

elsa_status elsa_cgne_solve(elsa_projector* p, const float* b, float* x, int32_t iterations,
                            int32_t useX0, void* stream)
{
    return guarded([&] {
        require(p && b && x && iterations >= 0, "elsa_cgne_solve: invalid argument");
        onDevice(p);
        elsa_b200::SolverWorkspace ws(p->impl->domainSize(), p->impl->rangeSize());
        elsa_b200::cgneSolve(*p->impl, b, x, iterations, useX0 != 0, ws, asStream(stream));
        ELSA_CUDA(cudaStreamSynchronize(asStream(stream)));
    });
}

elsa_status elsa_batch_cgne_create(elsa_projector* const* projectors, const float* const* b,
                                   float* const* x, int32_t count, void* stream,
                                   elsa_batch_cgne** out)
{
    return guarded([&] {
        require(out != nullptr, "elsa_batch_cgne_create: null output handle");
        *out = nullptr;
        require(count > 0 && projectors && b && x, "elsa_batch_cgne_create: invalid argument");
        std::vector<elsa_b200::Projector*> ops;
        std::vector<const float*> bs;
        std::vector<float*> xs;
        for (int32_t i = 0; i < count; ++i) {
            require(projectors[i] && b[i] && x[i], "elsa_batch_cgne_create: null instance");
            require(projectors[i]->impl->device() == projectors[0]->impl->device(),
                    "elsa_batch_cgne_create: all projectors must be on one device");
            ops.push_back(projectors[i]->impl.get());
            bs.push_back(b[i]);
            xs.push_back(x[i]);
        }
        onDevice(projectors[0]);
        auto h = std::make_unique<elsa_batch_cgne>();
        h->device = projectors[0]->impl->device();
        h->impl = std::make_unique<elsa_b200::BatchedCgne>(ops, bs, xs, asStream(stream));
        *out = h.release();
    });
}

namespace
{
    void onBatchDevice(const elsa_batch_cgne* h)
    {
        int cur = 0;
        ELSA_CUDA(cudaGetDevice(&cur));
        if (cur != h->device)
            ELSA_CUDA(cudaSetDevice(h->device));
    }
} // namespace

elsa_status elsa_batch_cgne_iterate(elsa_batch_cgne* h, int32_t iterations, void* stream)
{
    return guarded([&] {
        require(h && iterations >= 0, "elsa_batch_cgne_iterate: invalid argument");
        onBatchDevice(h);
        h->impl->iterate(iterations, asStream(stream));
    });
}

elsa_status elsa_batch_cgne_iterate_graph(elsa_batch_cgne* h, int32_t iterations, void* stream)
{
    return guarded([&] {
        require(h && iterations >= 0, "elsa_batch_cgne_iterate_graph: invalid argument");
        onBatchDevice(h);
        h->impl->iterateGraph(iterations, asStream(stream));
    });
}

elsa_status elsa_batch_cgne_residuals(elsa_batch_cgne* h, double* out, void* stream)
{
    return guarded([&] {
        require(h && out, "elsa_batch_cgne_residuals: null argument");
        onBatchDevice(h);
        h->impl->squaredResiduals(out, asStream(stream));
    });
}

elsa_status elsa_batch_cgne_destroy(elsa_batch_cgne* h)
{
    return guarded([&] {
        if (h) {
            onBatchDevice(h);
            ELSA_CUDA(cudaDeviceSynchronize()); // nothing in flight uses the workspaces
        }
        delete h;
    });
}

elsa_status elsa_cgne_split_create(elsa_projector* p, float* x, elsa_cgne_split** out)
{
    return guarded([&] {
        require(out != nullptr, "elsa_cgne_split_create: null output handle");
        *out = nullptr;
        require(p && x, "elsa_cgne_split_create: null argument");
        onDevice(p);
        auto h = std::make_unique<elsa_cgne_split>();
        h->device = p->impl->device();
        h->impl = std::make_unique<elsa_b200::SplitCgne>(*p->impl, x);
        *out = h.release();
    });
}

namespace
{
    void onSplitDevice(const elsa_cgne_split* c)
    {
        int cur = 0;
        ELSA_CUDA(cudaGetDevice(&cur));
        if (cur != c->device)
            ELSA_CUDA(cudaSetDevice(c->device));
    }
} // namespace

elsa_status elsa_cgne_split_backproject(elsa_cgne_split* c, const float* b, float* atb,
                                        void* stream)
{
    return guarded([&] {
        require(c && b && atb, "elsa_cgne_split_backproject: null argument");
        onSplitDevice(c);
        c->impl->backprojectData(b, atb, asStream(stream));
    });
}

elsa_status elsa_cgne_split_begin(elsa_cgne_split* c, const float* atb, void* stream)
{
    return guarded([&] {
        require(c && atb, "elsa_cgne_split_begin: null argument");
        onSplitDevice(c);
        c->impl->begin(atb, asStream(stream));
    });
}

elsa_status elsa_cgne_split_normal(elsa_cgne_split* c, float* q, void* stream)
{
    return guarded([&] {
        require(c && q, "elsa_cgne_split_normal: null argument");
        onSplitDevice(c);
        c->impl->applyNormal(q, asStream(stream));
    });
}

elsa_status elsa_cgne_split_update(elsa_cgne_split* c, const float* q, void* stream)
{
    return guarded([&] {
        require(c && q, "elsa_cgne_split_update: null argument");
        onSplitDevice(c);
        c->impl->update(q, asStream(stream));
    });
}

elsa_status elsa_cgne_split_residual(const elsa_cgne_split* c, double* result, void* stream)
{
    return guarded([&] {
        require(c && result, "elsa_cgne_split_residual: null argument");
        ELSA_CUDA(cudaMemcpyAsync(result, c->impl->squaredResidualDevice(), sizeof(double),
                                  cudaMemcpyDeviceToDevice, asStream(stream)));
    });
}

elsa_status elsa_cgne_split_destroy(elsa_cgne_split* c)
{
    return guarded([&] {
        if (c) {
            onSplitDevice(c);
            ELSA_CUDA(cudaDeviceSynchronize()); // no update in flight uses the workspace
        }
        delete c;
    });
}

elsa_status elsa_solver_create(int32_t kind, elsa_projector* p, const float* b, float* x,
                               int32_t useX0, const double* params, int32_t numParams,
                               void* stream, elsa_solver** out)
{
    return guarded([&] {
        require(out != nullptr, "elsa_solver_create: null output handle");
        *out = nullptr;
        require(p && b && x, "elsa_solver_create: null argument");
        require(kind >= ELSA_SOLVER_CGNE && kind <= ELSA_SOLVER_SQS,
                "elsa_solver_create: unknown solver kind");
        require(numParams >= 0 && (numParams == 0 || params != nullptr),
                "elsa_solver_create: invalid parameter array");
        static const int kMaxParams[] = {0, 2, 1, 6, 1, 1, 1, 2};
        require(numParams <= kMaxParams[kind], "elsa_solver_create: too many parameters");
        auto param = [&](int i, double dflt) { return i < numParams ? params[i] : dflt; };
        elsa_b200::SolverOptions opt;
        switch (kind) {
        case ELSA_SOLVER_CGLS:
            opt.cglsEps = param(0, 0.0);
            opt.cglsTol = param(1, 1e-4);
            require(std::isfinite(opt.cglsEps) && std::isfinite(opt.cglsTol),
                    "elsa_solver_create: CGLS eps and tol must be finite");
            break;
        case ELSA_SOLVER_LANDWEBER:
            opt.landweberStep = param(0, 0.0);
            require(std::isfinite(opt.landweberStep),
                    "elsa_solver_create: Landweber step must be finite");
            break;
        case ELSA_SOLVER_APGD: {
            opt.apgdMu = param(0, 0.0);
            opt.apgdEpsilon = param(1, static_cast<double>(FLT_EPSILON));
            const double prox = param(2, 0.0);
            require(prox == 0.0 || prox == 1.0 || prox == 2.0,
                    "elsa_solver_create: APGD proximal operator must be 0, 1 or 2");
            opt.prox.kind = static_cast<int>(prox);
            const double lo = param(3, std::nan("")), hi = param(4, std::nan(""));
            opt.prox.flags = (std::isnan(lo) ? 0 : 1) | (std::isnan(hi) ? 0 : 2);
            opt.prox.lo = std::isnan(lo) ? 0.0f : static_cast<float>(lo);
            opt.prox.hi = std::isnan(hi) ? 0.0f : static_cast<float>(hi);
            opt.prox.sigma = static_cast<float>(param(5, 1.0));
            require(std::isfinite(opt.apgdMu) && std::isfinite(opt.apgdEpsilon) &&
                        std::isfinite(opt.prox.sigma),
                    "elsa_solver_create: APGD parameters must be finite");
            if (opt.prox.kind == 1 && (opt.prox.flags & 3) == 3)
                require(opt.prox.lo <= opt.prox.hi,
                        "elsa_solver_create: box constraint with lower > upper");
            break;
        }
        case ELSA_SOLVER_SIRT:
            opt.sirtStep = param(0, 0.0);
            require(std::isfinite(opt.sirtStep), "elsa_solver_create: SIRT step must be finite");
            break;
        case ELSA_SOLVER_FGM:
        case ELSA_SOLVER_OGM:
            opt.momentumEpsilon = param(0, static_cast<double>(FLT_EPSILON));
            require(std::isfinite(opt.momentumEpsilon) && opt.momentumEpsilon >= 0.0,
                    "elsa_solver_create: epsilon must be finite and >= 0");
            break;
        case ELSA_SOLVER_SQS: {
            const double momentum = param(0, 1.0);
            require(momentum == 0.0 || momentum == 1.0,
                    "elsa_solver_create: SQS momentum must be 0 or 1");
            opt.sqsMomentum = momentum == 1.0;
            opt.sqsEpsilon = param(1, static_cast<double>(FLT_EPSILON));
            require(std::isfinite(opt.sqsEpsilon) && opt.sqsEpsilon >= 0.0,
                    "elsa_solver_create: epsilon must be finite and >= 0");
            break;
        }
        default:
            break;
        }
        onDevice(p);
        auto h = std::make_unique<elsa_solver>();
        h->device = p->impl->device();
        h->impl = std::make_unique<elsa_b200::SolverSession>(
            static_cast<elsa_b200::SolverKind>(kind), *p->impl, b, x, useX0 != 0, opt,
            asStream(stream));
        *out = h.release();
    });
}

elsa_status elsa_sqs_create(elsa_projector* p, const float* b,
                            elsa_projector* const* subsetProjectors, const float* const* subsetB,
                            int32_t numSubsets, float* x, int32_t useX0, int32_t momentum,
                            double epsilon, const float* preconditioner, void* stream,
                            elsa_solver** out)
{
    return guarded([&] {
        require(out != nullptr, "elsa_sqs_create: null output handle");
        *out = nullptr;
        require(p && b && x, "elsa_sqs_create: null argument");
        require(numSubsets == 0 || numSubsets >= 2,
                "elsa_sqs_create: use 0 subsets (full problem) or at least 2");
        require(numSubsets == 0 || (subsetProjectors && subsetB),
                "elsa_sqs_create: null subset arrays");
        require(momentum == 0 || momentum == 1, "elsa_sqs_create: momentum must be 0 or 1");
        require(std::isfinite(epsilon) && epsilon >= 0.0,
                "elsa_sqs_create: epsilon must be finite and >= 0");
        std::vector<elsa_b200::SubsetRef> subsets;
        for (int32_t i = 0; i < numSubsets; ++i) {
            require(subsetProjectors[i] && subsetB[i], "elsa_sqs_create: null subset");
            subsets.push_back({subsetProjectors[i]->impl.get(), subsetB[i]});
        }
        elsa_b200::SolverOptions opt;
        opt.sqsMomentum = momentum != 0;
        opt.sqsEpsilon = epsilon;
        opt.sqsPreconditioner = preconditioner;
        onDevice(p);
        auto h = std::make_unique<elsa_solver>();
        h->device = p->impl->device();
        h->impl = std::make_unique<elsa_b200::SolverSession>(
            elsa_b200::SolverKind::SQS, *p->impl, b, x, useX0 != 0, opt, asStream(stream),
            std::move(subsets));
        *out = h.release();
    });
}

elsa_status elsa_subset_split(int32_t dim, const float* poses, int32_t numPoses,
                              int32_t numSubsets, int32_t strategy, int32_t* viewOrder,
                              int32_t* subsetSizes)
{
    return guarded([&] {
        require(poses && viewOrder && subsetSizes, "elsa_subset_split: null argument");
        require(dim == 2 || dim == 3, "elsa_subset_split: dim must be 2 or 3");
        require(numPoses >= 1, "elsa_subset_split: no poses");
        require(numSubsets >= 2, "SubsetSampler: nSubsets must be >= 2");
        require(strategy == ELSA_SUBSET_ROUND_ROBIN ||
                    strategy == ELSA_SUBSET_ROTATIONAL_CLUSTERING,
                "SubsetSampler: unsupported sampling strategy");
        std::vector<elsa_b200::PoseRecord> recs(static_cast<size_t>(numPoses));
        std::memcpy(recs.data(), poses, sizeof(float) * elsa_b200::kPoseFloats * recs.size());
        std::vector<std::vector<int>> parts;
        if (strategy == ELSA_SUBSET_ROUND_ROBIN) {
            std::vector<int> idx(static_cast<size_t>(numPoses));
            for (int32_t i = 0; i < numPoses; ++i)
                idx[static_cast<size_t>(i)] = i;
            parts = elsa_b200::splitRoundRobin(idx, numSubsets);
        } else {
            parts = elsa_b200::splitRotationalClustering(dim, recs, numSubsets);
        }
        int32_t k = 0;
        for (int32_t i = 0; i < numSubsets; ++i) {
            const auto& part = parts[static_cast<size_t>(i)];
            subsetSizes[i] = static_cast<int32_t>(part.size());
            for (int v : part)
                viewOrder[k++] = v;
        }
    });
}

elsa_status elsa_gather_views(const float* sinogram, int64_t viewSize, const int32_t* viewOrder,
                              int32_t numViews, int32_t totalViews, float* out, void* stream)
{
    return guarded([&] {
        require(viewSize >= 0 && numViews >= 0 && totalViews >= 0,
                "elsa_gather_views: negative size");
        require(numViews == 0 || viewSize == 0 || (sinogram && out && viewOrder),
                "elsa_gather_views: null argument");
        for (int32_t j = 0; j < numViews; ++j) {
            const int32_t v = viewOrder[j];
            require(v >= 0 && v < totalViews, "elsa_gather_views: view index out of range");
        }
        for (int32_t j = 0; j < numViews && viewSize > 0; ++j)
            ELSA_CUDA(cudaMemcpyAsync(out + static_cast<int64_t>(j) * viewSize,
                                      sinogram + static_cast<int64_t>(viewOrder[j]) * viewSize,
                                      sizeof(float) * static_cast<size_t>(viewSize),
                                      cudaMemcpyDeviceToDevice, asStream(stream)));
    });
}

elsa_status elsa_solver_step_size(elsa_solver* s, double* value)
{
    return guarded([&] {
        require(s && value, "elsa_solver_step_size: null argument");
        *value = s->impl->stepSize();
    });
}

elsa_status elsa_power_iterations(elsa_projector* p, int32_t iterations, void* stream,
                                  double* value)
{
    return guarded([&] {
        require(p && value && iterations >= 0, "elsa_power_iterations: invalid argument");
        onDevice(p);
        elsa_b200::SolverWorkspace ws(p->impl->domainSize(), p->impl->rangeSize());
        *value = elsa_b200::powerIterationsAtA(*p->impl, ws, iterations, asStream(stream));
    });
}

elsa_status elsa_solver_iterate(elsa_solver* s, int32_t iterations, void* stream)
{
    return guarded([&] {
        require(s && iterations >= 0, "elsa_solver_iterate: invalid argument");
        ELSA_CUDA(cudaSetDevice(s->device));
        s->impl->iterate(iterations, asStream(stream));
    });
}

elsa_status elsa_solver_iterate_graph(elsa_solver* s, int32_t iterations, void* stream)
{
    return guarded([&] {
        require(s && iterations >= 0, "elsa_solver_iterate_graph: invalid argument");
        ELSA_CUDA(cudaSetDevice(s->device));
        s->impl->iterateGraph(iterations, asStream(stream));
    });
}

elsa_status elsa_solve_batch(elsa_solver* const* solvers, int32_t n, int32_t iterations,
                             int32_t numStreams)
{
    return guarded([&] {
        require(n >= 0 && (n == 0 || solvers) && iterations >= 0 && numStreams >= 1 &&
                    numStreams <= 64,
                "elsa_solve_batch: invalid argument");
        std::vector<elsa_b200::SolverSession*> sessions(static_cast<size_t>(n));
        for (int i = 0; i < n; ++i) {
            require(solvers[i] != nullptr, "elsa_solve_batch: null solver");
            require(solvers[i]->device == solvers[0]->device,
                    "elsa_solve_batch: solvers on different devices");
            sessions[static_cast<size_t>(i)] = solvers[i]->impl.get();
        }
        if (n > 0)
            ELSA_CUDA(cudaSetDevice(solvers[0]->device));
        elsa_b200::solveBatch(sessions.data(), n, iterations, numStreams);
    });
}

elsa_status elsa_solver_squared_residual(elsa_solver* s, void* stream, double* value)
{
    return guarded([&] {
        require(s && value, "elsa_solver_squared_residual: null argument");
        ELSA_CUDA(cudaSetDevice(s->device));
        *value = s->impl->squaredResidual(asStream(stream));
    });
}

elsa_status elsa_solver_enable_timing(elsa_solver* s, int32_t enable)
{
    return guarded([&] {
        require(s != nullptr, "elsa_solver_enable_timing: null argument");
        s->impl->timer().enable(enable != 0);
    });
}

elsa_status elsa_solver_timing(elsa_solver* s, double* fwd, double* adj, int64_t* count)
{
    return guarded([&] {
        require(s && fwd && adj && count, "elsa_solver_timing: null argument");
        ELSA_CUDA(cudaSetDevice(s->device));
        s->impl->timer().collect(*fwd, *adj, *count);
    });
}

elsa_status elsa_solver_destroy(elsa_solver* s)
{
    return guarded([&] { delete s; });
}

} // extern "C"

namespace
{
    void fillInfo(const elsa_b200::io::ImageInfo& in, elsa_image_info* out)
    {
        if (in.dims.size() > ELSA_IO_MAX_DIMS)
            throw elsa_b200::Error(ELSA_ERROR_NOT_SUPPORTED, "image has too many dimensions");
        std::memset(out, 0, sizeof(*out));
        out->ndim = static_cast<int32_t>(in.dims.size());
        out->data_type = static_cast<int32_t>(in.type);
        for (size_t i = 0; i < in.dims.size(); ++i) {
            out->dims[i] = in.dims[i];
            out->spacing[i] = in.spacing[i];
        }
    }

    std::vector<int64_t> shapeOf(int32_t ndim, const int64_t* dims, const char* who)
    {
        require(ndim >= 1 && ndim <= ELSA_IO_MAX_DIMS && dims != nullptr, who);
        return std::vector<int64_t>(dims, dims + ndim);
    }

    std::vector<float> spacingOf(int32_t ndim, const float* spacing)
    {
        return spacing ? std::vector<float>(spacing, spacing + ndim)
                       : std::vector<float>(static_cast<size_t>(ndim), 1.0f);
    }
} // namespace

extern "C" {

elsa_status elsa_edf_info(const char* path, elsa_image_info* info)
{
    return guarded([&] {
        require(path && info, "elsa_edf_info: null argument");
        fillInfo(elsa_b200::io::edfInfo(path), info);
    });
}

elsa_status elsa_edf_read(const char* path, float* out, int64_t count)
{
    return guarded([&] {
        require(path && (out || count == 0) && count >= 0, "elsa_edf_read: invalid argument");
        elsa_b200::io::edfRead(path, out, count);
    });
}

elsa_status elsa_edf_write(const char* path, const float* data, int32_t ndim, const int64_t* dims,
                           const float* spacing)
{
    return guarded([&] {
        require(path && data, "elsa_edf_write: null argument");
        elsa_b200::io::edfWrite(path, data, shapeOf(ndim, dims, "elsa_edf_write: bad shape"),
                                spacingOf(ndim, spacing));
    });
}

elsa_status elsa_mhd_info(const char* metaPath, elsa_image_info* info)
{
    return guarded([&] {
        require(metaPath && info, "elsa_mhd_info: null argument");
        fillInfo(elsa_b200::io::mhdInfo(metaPath), info);
    });
}

elsa_status elsa_mhd_read(const char* metaPath, float* out, int64_t count)
{
    return guarded([&] {
        require(metaPath && (out || count == 0) && count >= 0, "elsa_mhd_read: invalid argument");
        elsa_b200::io::mhdRead(metaPath, out, count);
    });
}

elsa_status elsa_mhd_write(const char* metaPath, const char* rawPath, const float* data,
                           int32_t ndim, const int64_t* dims, const float* spacing)
{
    return guarded([&] {
        require(metaPath && rawPath && data, "elsa_mhd_write: null argument");
        elsa_b200::io::mhdWrite(metaPath, rawPath, data,
                                shapeOf(ndim, dims, "elsa_mhd_write: bad shape"),
                                spacingOf(ndim, spacing));
    });
}

elsa_status elsa_pgm_write(const char* path, const float* data, int32_t ndim, const int64_t* dims)
{
    return guarded([&] {
        require(path && data, "elsa_pgm_write: null argument");
        elsa_b200::io::pgmWrite(path, data, shapeOf(ndim, dims, "elsa_pgm_write: bad shape"));
    });
}

} // extern "C"
