// Autotuner of the projectors' launch parameters (see tune.hpp).
#include "tune.hpp"

#include <algorithm>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>

#include "solvers.hpp"

namespace elsa_b200
{
    void Projector::setKnob(int knob, int value)
    {
        (void)value;
        throw Error(ELSA_ERROR_NOT_SUPPORTED,
                    "projector knob " + std::to_string(knob) + " is not tunable here");
    }

    std::vector<int> chunkCandidates(int limit, int extra)
    {
        std::vector<int> c;
        for (int v = 1; v <= limit; v *= 2)
            c.push_back(v);
        if (extra >= 1 && extra <= limit)
            c.push_back(extra);
        std::sort(c.begin(), c.end());
        c.erase(std::unique(c.begin(), c.end()), c.end());
        return c;
    }

    namespace
    {
        std::mutex gCacheMutex;
        std::map<std::string, KnobValues>& cache()
        {
            static std::map<std::string, KnobValues> c;
            return c;
        }

        bool validKey(const std::string& key)
        {
            if (key.empty())
                return false;
            for (char ch : key)
                if (ch == ' ' || ch == '\t' || ch == '\n' || ch == '\r')
                    return false;
            return true;
        }

        // Mean milliseconds of `reps` calls of `op` after one untimed call.
        template <class Op>
        double timeOp(Op&& op, cudaStream_t s, int reps)
        {
            cudaEvent_t a, b;
            ELSA_CUDA(cudaEventCreate(&a));
            ELSA_CUDA(cudaEventCreate(&b));
            op();
            ELSA_CUDA(cudaEventRecord(a, s));
            for (int i = 0; i < reps; ++i)
                op();
            ELSA_CUDA(cudaEventRecord(b, s));
            ELSA_CUDA(cudaEventSynchronize(b));
            float ms = 0.0f;
            ELSA_CUDA(cudaEventElapsedTime(&ms, a, b));
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            return static_cast<double>(ms) / reps;
        }
    } // namespace

    std::string tuneKey(const Projector& p)
    {
        std::ostringstream k;
        const VolumeShape& v = p.volume();
        const DetectorShape& d = p.detector();
        k << p.kind() << ':' << v.dim << ':' << v.n[0] << ',' << v.n[1] << ',' << v.n[2] << ':'
          << d.nu << ',' << d.nv << ',' << d.np;
        return k.str();
    }

    TuneResult autotune(Projector& p, cudaStream_t s, bool force)
    {
        TuneResult res;
        const std::string key = tuneKey(p);
        KnobValues cached{};
        if (!force && tuneCacheGet(key, cached)) {
            for (int k = 0; k < kKnobCount; ++k) {
                const std::vector<int> cand = p.knobCandidates(k);
                if (cached[k] >= 0 && std::find(cand.begin(), cand.end(), cached[k]) != cand.end())
                    p.setKnob(k, cached[k]);
                res.values[k] = p.knob(k);
            }
            res.fromCache = true;
            ELSA_CUDA(cudaStreamSynchronize(s));
            return res;
        }
        // scratch operands: the kernels' run time does not depend on the values
        DeviceBuffer x(sizeof(float) * static_cast<size_t>(p.domainSize()));
        DeviceBuffer y(sizeof(float) * static_cast<size_t>(p.rangeSize()));
        ELSA_CUDA(cudaMemsetAsync(x.as<float>(), 0, x.bytes(), s));
        ELSA_CUDA(cudaMemsetAsync(y.as<float>(), 0, y.bytes(), s));
        auto fwd = [&] { p.forward(x.as<float>(), y.as<float>(), s); };
        auto adj = [&] { p.adjoint(y.as<float>(), x.as<float>(), s); };
        constexpr int kReps = 3;
        for (int k = 0; k < kKnobCount; ++k) {
            const std::vector<int> cand = p.knobCandidates(k);
            if (cand.empty()) {
                res.values[k] = p.knob(k);
                continue;
            }
            const bool forwardKnob = k == kKnobForwardThreads;
            int best = p.knob(k);
            double bestMs = -1.0;
            for (int v : cand) {
                p.setKnob(k, v);
                const double ms = forwardKnob ? timeOp(fwd, s, kReps) : timeOp(adj, s, kReps);
                if (bestMs < 0.0 || ms < bestMs) {
                    bestMs = ms;
                    best = v;
                }
            }
            p.setKnob(k, best);
            res.values[k] = best;
            if (forwardKnob)
                res.forwardMs = bestMs;
            else
                res.adjointMs = res.adjointMs > 0.0 ? std::min(res.adjointMs, bestMs) : bestMs;
        }
        ELSA_CUDA(cudaStreamSynchronize(s));
        tuneCachePut(key, res.values);
        return res;
    }

    void tuneCacheClear()
    {
        std::lock_guard<std::mutex> g(gCacheMutex);
        cache().clear();
    }

    size_t tuneCacheSize()
    {
        std::lock_guard<std::mutex> g(gCacheMutex);
        return cache().size();
    }

    bool tuneCacheGet(const std::string& key, KnobValues& values)
    {
        std::lock_guard<std::mutex> g(gCacheMutex);
        auto it = cache().find(key);
        if (it == cache().end())
            return false;
        values = it->second;
        return true;
    }

    void tuneCachePut(const std::string& key, const KnobValues& values)
    {
        if (!validKey(key))
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "tune cache: invalid key");
        std::lock_guard<std::mutex> g(gCacheMutex);
        cache()[key] = values;
    }

    void tuneCacheSave(const std::string& path)
    {
        std::ostringstream out;
        {
            std::lock_guard<std::mutex> g(gCacheMutex);
            for (const auto& kv : cache()) {
                out << kv.first;
                for (int v : kv.second)
                    out << ' ' << v;
                out << '\n';
            }
        }
        std::ofstream f(path, std::ios::trunc);
        if (!f)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "tune cache: cannot write " + path);
        f << out.str();
        if (!f)
            throw Error(ELSA_ERROR_LOGIC, "tune cache: write failed for " + path);
    }

    void tuneCacheLoad(const std::string& path)
    {
        std::ifstream f(path);
        if (!f)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "tune cache: cannot read " + path);
        std::vector<std::pair<std::string, KnobValues>> entries;
        std::string line;
        int lineNo = 0;
        while (std::getline(f, line)) {
            ++lineNo;
            if (line.empty())
                continue;
            std::istringstream in(line);
            std::string key;
            KnobValues v{};
            in >> key;
            for (int k = 0; k < kKnobCount; ++k)
                if (!(in >> v[k]) || v[k] < -1)
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                                "tune cache: bad entry on line " + std::to_string(lineNo));
            std::string rest;
            if (in >> rest || !validKey(key))
                throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                            "tune cache: bad entry on line " + std::to_string(lineNo));
            entries.emplace_back(key, v);
        }
        std::lock_guard<std::mutex> g(gCacheMutex);
        for (const auto& e : entries)
            cache()[e.first] = e.second;
    }
} // namespace elsa_b200
