// Exercises the C++ layer (include/elsa_b200.hpp) the way elsa's examples use elsa
// (examples/example3d.cpp): trajectory, projector, forward projection, CGNE, CGLS, APGD, SIRT,
// FGM, OGM, SQS (plain, ordered subsets, preconditioned), the BinaryMethod and ray-driven LUT
// projectors, a curved detector, the autotuner and the image files. Writes the sinogram, the
// projections and the reconstructions as raw float32 files into the directory given as the first
// argument, and prints one line of residuals.
#include <cstdio>
#include <fstream>
#include <string>

#include "elsa_b200.hpp"

using namespace elsa_b200::elsa;

static void save(const std::string& path, const std::vector<float>& v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * 4));
}

int main(int argc, char** argv)
{
    const std::string dir = argc > 1 ? argv[1] : ".";
    try {
        auto vol = std::make_shared<VolumeDescriptor>(IndexVector{24, 24, 24});
        auto sino = CircleTrajectoryGenerator::createTrajectory(30, *vol, 360, 240.0f, 60.0f,
                                                                IndexVector{36, 36});
        // a centred cube of ones as the phantom
        std::vector<float> phantom(24 * 24 * 24, 0.0f);
        for (int z = 6; z < 18; ++z)
            for (int y = 6; y < 18; ++y)
                for (int x = 6; x < 18; ++x)
                    phantom[x + 24 * (y + 24 * z)] = 1.0f;
        DataContainer<float> x(vol, phantom);
        JosephsMethodCUDA<float> A(*vol, *sino);
        DataContainer<float> b = A.apply(x);
        save(dir + "/sino.f32", b.toHost());
        save(dir + "/poses.f32", sino->poses());

        CGNE<float> cgne(A, b);
        auto r1 = cgne.solve(8);
        CGLS<float> cgls(A, b);
        auto r2 = cgls.solve(8);
        APGD<float> apgd(A, b, ProximalBoxConstraint{0.0f, std::nullopt});
        auto r3 = apgd.solve(8);
        save(dir + "/cgne.f32", r1.toHost());
        save(dir + "/cgls.f32", r2.toHost());
        save(dir + "/apgd.f32", r3.toHost());

        // SIRT, FGM, OGM on the same problem
        save(dir + "/sirt.f32", SIRT<float>(A, b).solve(6).toHost());
        save(dir + "/fgm.f32", FGM<float>(LeastSquares<float>{A, b}).solve(6).toHost());
        save(dir + "/ogm.f32", OGM<float>(LeastSquares<float>{A, b}).solve(6).toHost());

        // SQS: full problem, then 3 round-robin subsets with a Scaling preconditioner
        save(dir + "/sqs.f32", SQS<float>(LeastSquares<float>{A, b}).solve(4).toHost());
        SubsetSampler<PlanarDetectorDescriptor, float> sampler(
            *vol, *sino, 3, SubsetSampler<PlanarDetectorDescriptor, float>::SamplingStrategy::
                                ROUND_ROBIN);
        auto blocks = sampler.getPartitionedData(b);
        auto subsetOps = sampler.getSubsetProjectors<JosephsMethodCUDA<float>>();
        std::vector<LeastSquares<float>> subsets;
        for (size_t i = 0; i < subsetOps.size(); ++i)
            subsets.push_back(LeastSquares<float>{*subsetOps[i], blocks[i]});
        std::vector<float> diag(24 * 24 * 24);
        for (size_t i = 0; i < diag.size(); ++i)
            diag[i] = 0.5f + 0.5f * static_cast<float>(i % 7) / 6.0f;
        DataContainer<float> precond(vol, diag);
        Scaling<float> scaling{precond};
        save(dir + "/sqs_os.f32",
             SQS<float>(LeastSquares<float>{A, b}, subsets, scaling).solve(3).toHost());
        for (size_t i = 0; i < blocks.size(); ++i)
            save(dir + "/block" + std::to_string(i) + ".f32", blocks[i].toHost());

        // Siddon with the atomic scatter adjoint, then with its bit-reproducible brick owner
        // (the default)
        SiddonsMethodCUDA<float> S(*vol, *sino);
        S.setKnob(ELSA_KNOB_ADJOINT_SCATTER, 1);
        const auto scatterAdj = S.applyAdjoint(b).toHost();
        S.setKnob(ELSA_KNOB_ADJOINT_SCATTER, 0);
        if (S.getKnob(ELSA_KNOB_ADJOINT_SCATTER) != 0)
            throw elsa_b200::Error(ELSA_ERROR_LOGIC, "knob not set");
        save(dir + "/siddon_adj_scatter.f32", scatterAdj);
        save(dir + "/siddon_adj_owner.f32", S.applyAdjoint(b).toHost());

        // BinaryMethod and the ray-driven blob / B-spline projectors (forward of the phantom)
        BinaryMethod<float> binary(*vol, *sino);
        save(dir + "/binary.f32", binary.apply(x).toHost());
        BlobProjector<float> blob(*vol, *sino);
        save(dir + "/rayblob.f32", blob.apply(x).toHost());
        BSplineProjector<float> bspline(*vol, *sino);
        save(dir + "/raybspline.f32", bspline.apply(x).toHost());

        // a curved detector (opening angle 0.6 rad), tuned before use
        auto curved = CurvedCircleTrajectoryGenerator::createTrajectory(
            30, *vol, 360, 240.0f, 60.0f, 0.6f, IndexVector{36, 36});
        JosephsMethodCUDA<float> Ac(*vol, *curved);
        Ac.autotune();
        const bool cached = Ac.autotune(); // the second call finds the geometry in the cache
        save(dir + "/curved.f32", Ac.apply(x).toHost());
        save(dir + "/curved_coords.f32", curved->getPlanarCoords());

        // JosephsMethodCUDA(..., fast = true): elsa's unmatched adjoint, the same forward
        JosephsMethodCUDA<float> Afast(*vol, *sino, true);
        if (Afast.apply(x).toHost() != b.toHost())
            throw elsa_b200::Error(ELSA_ERROR_LOGIC, "fast flag changed the forward");
        save(dir + "/fast_adjoint.f32", Afast.applyAdjoint(b).toHost());
        save(dir + "/matched_adjoint.f32", JosephsMethod<float>(*vol, *sino).applyAdjoint(b).toHost());

        // image files: the sinogram through EDF and MHD, a slice as PGM
        EDF::write(b, dir + "/sino.edf");
        MHD::write(b, dir + "/sino.mhd", dir + "/sino.raw");
        const auto fromEdf = EDF::read<float>(dir + "/sino.edf").toHost();
        const auto fromMhd = MHD::read<float>(dir + "/sino.mhd").toHost();
        const auto ref = b.toHost();
        if (fromEdf != ref || fromMhd != ref)
            throw elsa_b200::Error(ELSA_ERROR_LOGIC, "image file round trip differs");
        auto sliceDesc = std::make_shared<VolumeDescriptor>(IndexVector{24, 24});
        std::vector<float> slice(phantom.begin() + 24 * 24 * 12, phantom.begin() + 24 * 24 * 13);
        PGM::write(DataContainer<float>(sliceDesc, slice), dir + "/slice.pgm");

        std::printf("ok %.6g %.6g %.6g %.6g %d\n", b.squaredL2Norm(), cgne.lastSquaredResidual(),
                    cgls.lastSquaredResidual(), powerIterations(A, 5), cached ? 1 : 0);
    } catch (const elsa_b200::Error& e) {
        std::fprintf(stderr, "error %d: %s\n", static_cast<int>(e.status), e.what());
        return 1;
    }
    return 0;
}
