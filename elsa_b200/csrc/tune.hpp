// Autotuner of the projectors' launch parameters (Knob in projector.hpp).
//
// autotune() times every candidate of every knob a projector offers (the forward for the
// forward knob, the adjoint for the adjoint knobs) with CUDA events on the caller's stream,
// keeps the fastest, and records the choice in a process-wide cache keyed by the projector kind
// and its volume and detector sizes, so that later projectors of the same shape take the cached
// values without timing. The cache can be written to and read from a text file (one line per
// key: the key, then one value per knob, -1 for knobs the projector does not use).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <string>

#include "projector.hpp"

namespace elsa_b200
{
    using KnobValues = std::array<int, kKnobCount>;

    struct TuneResult {
        KnobValues values{};
        bool fromCache = false;
        double forwardMs = 0.0; // best forward time seen (0 when taken from the cache)
        double adjointMs = 0.0; // best adjoint time seen (0 when taken from the cache)
    };

    // Cache key: "kind:dim:nx,ny,nz:nu,nv,np".
    std::string tuneKey(const Projector& p);

    // Tune `p` (or apply the cached values of its key unless `force`). Synchronizes `stream`.
    TuneResult autotune(Projector& p, cudaStream_t stream, bool force);

    void tuneCacheClear();
    size_t tuneCacheSize();
    bool tuneCacheGet(const std::string& key, KnobValues& values);
    void tuneCachePut(const std::string& key, const KnobValues& values);
    // Write every entry to `path` (replacing the file); read entries from `path`, adding to or
    // replacing the cached ones. Both throw elsa_b200::Error on I/O or format errors.
    void tuneCacheSave(const std::string& path);
    void tuneCacheLoad(const std::string& path);
} // namespace elsa_b200
