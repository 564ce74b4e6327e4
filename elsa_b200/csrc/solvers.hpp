// Device solvers and their scratch buffers.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "projector.hpp"
#include "vecops.cuh"

namespace elsa_b200
{
    class DeviceBuffer
    {
    public:
        DeviceBuffer() = default;
        explicit DeviceBuffer(size_t bytes);
        ~DeviceBuffer();
        DeviceBuffer(const DeviceBuffer&) = delete;
        DeviceBuffer& operator=(const DeviceBuffer&) = delete;
        template <typename T>
        T* as() const
        {
            return static_cast<T*>(ptr_);
        }
        size_t bytes() const { return bytes_; }

    private:
        void* ptr_ = nullptr;
        size_t bytes_ = 0;
    };

    // Scratch for one solver run: four volume-sized and one sinogram-sized float buffers, the
    // reduction partials and the device scalars.
    struct SolverWorkspace {
        SolverWorkspace(int64_t domain, int64_t range);
        DeviceBuffer vol0, vol1, vol2, vol3, sino0, partials, scalars;
    };

    void cgneSolve(Projector& A, const float* b, float* x, int iterations, bool useX0,
                   SolverWorkspace& ws, cudaStream_t s);
    void cgneIteration(Projector& A, float* x, float* r, float* c, float* q, float* sino,
                       double* partials, SolverScalars* S, cudaStream_t s);
} // namespace elsa_b200
