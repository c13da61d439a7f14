// flip2_main -- the reference's engine/main.cu driver loop written against the
// C++ facade: random initial positions in the lower-middle of the domain
// (engine/testing.h:55-76, here seeded), initialize, then solveFrame at
// 24 fps with a CSV of positions after each frame.
//
//   flip2_main [particles] [frames] [native|reference] [outdir]
//
// With outdir, frame f is written as outdir/f (the reference's "x, y, z" CSV)
// and outdir/f.bin (exact FP32 positions), and the initial x coordinates go
// through a CudaVec<double> and its getMax: outdir/px0.f64 holds them (raw
// doubles) and outdir/getmax.txt the device maximum of their absolute values
// (%.17g).
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include "flip2/particles.hpp"

int main(int argc, char** argv) {
    unsigned n = argc > 1 ? (unsigned)std::strtoul(argv[1], nullptr, 10) : (1u << 19) - 24u;
    int frames = argc > 2 ? std::atoi(argv[2]) : 3;
    bool native = argc > 3 ? std::string(argv[3]) != "reference" : true;
    std::string outdir = argc > 4 ? argv[4] : "";
    try {
        flip2::Particles particles(n, native ? FLIP_MODE_NATIVE : FLIP_MODE_REFERENCE);
        // native mode needs 4*size % 8 == 0: 64 root cells of 0.25 (the reference uses 100)
        unsigned R = native ? 64 : 100;
        particles.setDomain(-10.0, -10.0, -10.0, R, R, R, 0.25);
        std::mt19937_64 rng(0);
        const flip2::Grid& g = particles.grid;
        double third = g.sizeY * g.cellSize / 3.0;
        std::uniform_real_distribution<> dx(g.negX + third, g.negX + g.sizeX * g.cellSize - third);
        std::uniform_real_distribution<> dy(g.negY, g.negY + g.sizeY * g.cellSize - third);
        std::uniform_real_distribution<> dz(g.negZ + third, g.negZ + g.sizeZ * g.cellSize - third);
        std::vector<double> px(n), py(n), pz(n), zero(n, 0.0);
        for (unsigned i = 0; i < n; ++i) { px[i] = dx(rng); py[i] = dy(rng); pz[i] = dz(rng); }
        particles.upload(px, py, pz, &zero, &zero, &zero);
        if (!outdir.empty()) {
            flip2::CudaVec<double> xs(n);
            for (unsigned i = 0; i < n; ++i) xs[i] = px[i];
            xs.upload();
            double m = xs.getMax(nullptr, true);
            FILE* f = std::fopen((outdir + "/getmax.txt").c_str(), "w");
            FILE* g = std::fopen((outdir + "/px0.f64").c_str(), "wb");
            if (!f || !g) throw flip2::Error(FLIP_ERR_ARG, "cannot write into " + outdir);
            std::fprintf(f, "%.17g\n", m);
            std::fwrite(px.data(), sizeof(double), n, g);
            std::fclose(f);
            std::fclose(g);
        }
        particles.initialize();
        if (!outdir.empty()) {
            particles.writePositionsToFile(outdir + "/0");
            particles.writePositionsToBinaryFile(outdir + "/0.bin");
        }
        for (int f = 0; f < frames; ++f) {
            particles.solveFrame(24.0);
            flip_info i = particles.info();
            std::printf("frame %d: t=%.5f dt=%.3g pressure iters %d residual %.3g\n", f + 1, i.elapsed_time, i.dt,
                        i.pressure_iters, i.residual);
            if (!outdir.empty()) {
                particles.writePositionsToFile(outdir + "/" + std::to_string(f + 1));
                particles.writePositionsToBinaryFile(outdir + "/" + std::to_string(f + 1) + ".bin");
            }
        }
    } catch (const flip2::Error& e) {
        std::fprintf(stderr, "flip2_main: %s\n", e.what());
        return 1;
    }
    return 0;
}
