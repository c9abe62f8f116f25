// beam_linear_static.cpp -- test driver: the call sequence of the reference's
// examples/beam_linear_static.cc (element set-up, mass, LinearStaticSolver,
// Solve, positions back) through the C++ classes of include/tlfea/tlfea.hpp.
//
// usage: beam_linear_static <in.bin> <out.bin>
//   in.bin : int32 N, E, n_fixed; double x[N], y[N], z[N];
//            int32 conn[E*10] (column-major); int32 fixed[n_fixed]; double f[3N]
//   out.bin: int32 iterations; double residual; double u[3N] (solved - reference positions)
// Exit codes: 0 solved, 1 bad input, 2 library error, 3 no CUDA device.
#include <cstdio>
#include <vector>

#include "tlfea/tlfea.hpp"

using namespace tlfea_cxx;

template <typename T>
static bool rd(FILE* f, T* p, size_t n) {
    return std::fread(p, sizeof(T), n, f) == n;
}

int main(int argc, char** argv) {
    if (argc != 3) return 1;
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 1;
    int N = 0, E = 0, nf = 0;
    if (!rd(in, &N, 1) || !rd(in, &E, 1) || !rd(in, &nf, 1) || N <= 0 || E <= 0 || nf < 0) return 1;
    VectorXR x(N), y(N), z(N), f(3 * (size_t)N);
    std::vector<int> conn(10 * (size_t)E), fixed(nf);
    if (!rd(in, x.data(), N) || !rd(in, y.data(), N) || !rd(in, z.data(), N) || !rd(in, conn.data(), conn.size()) ||
        !rd(in, fixed.data(), fixed.size()) || !rd(in, f.data(), f.size()))
        return 1;
    std::fclose(in);

    GPU_FEAT10_Data beam(E, N);
    beam.Initialize();
    if (!beam.handle()) {
        std::fprintf(stderr, "no CUDA device\n");
        return 3;
    }
    // Keast 5-point rule (quadrature_utils.h:125-160)
    const double a = 0.5, c = 1.0 / 6.0;
    VectorXR qx = {0.25, c, a, c, c}, qy = {0.25, c, c, a, c}, qz = {0.25, c, c, c, a};
    VectorXR qw = {-0.8 / 6.0, 0.45 / 6.0, 0.45 / 6.0, 0.45 / 6.0, 0.45 / 6.0};
    beam.SetNodalFixed(fixed);
    beam.SetExternalForce(f);
    beam.Setup(qx, qy, qz, qw, x, y, z, conn);
    beam.SetDensity(1000.0);
    beam.SetDamping(0.0, 0.0);
    beam.SetSVK(1e7, 0.3);
    beam.CalcDnDuPre();
    beam.CalcMassMatrix();

    FEASolver fea;
    fea.AddElement("beam", &beam);
    LinearStaticSolver<GPU_FEAT10_Data> solver(&beam, 1e-10, 50000);
    fea.AddSolver("static", &solver);
    fea.GetSolver("static")->Solve();

    VectorXR x2, y2, z2;
    beam.RetrievePositionToCPU(x2, y2, z2);
    VectorXR u(3 * (size_t)N);
    for (int i = 0; i < N; ++i) {
        u[3 * i + 0] = x2[i] - x[i];
        u[3 * i + 1] = y2[i] - y[i];
        u[3 * i + 2] = z2[i] - z[i];
    }
    const int it = solver.GetLastIterCount();
    const double res = solver.GetLastResidual();
    beam.Destroy();
    if (it <= 0) return 2;
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 1;
    std::fwrite(&it, sizeof(int), 1, out);
    std::fwrite(&res, sizeof(double), 1, out);
    std::fwrite(u.data(), sizeof(double), u.size(), out);
    std::fclose(out);
    std::printf("iterations %d residual %.3e\n", it, res);
    return 0;
}
