// Exercises the C++ layer (include/elsa_b200.hpp) the way elsa's examples use elsa
// (examples/example3d.cpp): trajectory, projector, forward projection, CGNE, CGLS, APGD.
// Writes the sinogram and the reconstructions as raw float32 files into the directory given as
// the first argument, and prints one line of residuals.
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
        std::printf("ok %.6g %.6g %.6g %.6g\n", b.squaredL2Norm(), cgne.lastSquaredResidual(),
                    cgls.lastSquaredResidual(), powerIterations(A, 5));
    } catch (const elsa_b200::Error& e) {
        std::fprintf(stderr, "error %d: %s\n", static_cast<int>(e.status), e.what());
        return 1;
    }
    return 0;
}
