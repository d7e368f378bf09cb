// Links the C++ drop-in interface (the reference's function names and
// signatures) against libgmxcorr_b200.so the way the reference front end
// would, and writes every estimator's matrix for tests/test_gpu_dropin.py.
//   dropin_check <coords.bin> <k> <lag> <out_prefix>
// coords.bin: int32 natoms, int32 nframes, then natoms*nframes*3 doubles.
#include "correlation_core.h"
#include "gcmi.h"
#include "kraskov_gpu.h"
#include "transfer_entropy.h"

#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

static void dump(const std::string& path, const std::vector<double>& m)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    std::fwrite(m.data(), sizeof(double), m.size(), f);
    std::fclose(f);
}

int main(int argc, char** argv)
{
    if (argc != 5)
        return 2;
    FILE* f = std::fopen(argv[1], "rb");
    int   n = 0, T = 0;
    if (std::fread(&n, 4, 1, f) != 1 || std::fread(&T, 4, 1, f) != 1)
        return 3;
    t_traj traj;
    traj.natoms  = n;
    traj.nframes = T;
    snew(traj.x, n);
    snew(traj.xav, n);
    for (int a = 0; a < n; ++a)
    {
        snew(traj.x[a], T);
        if (std::fread(traj.x[a], sizeof(double), (size_t)3 * T, f) != (size_t)3 * T)
            return 4;
    }
    std::fclose(f);
    const int         k = std::atoi(argv[2]), lag = std::atoi(argv[3]);
    const std::string pre = argv[4];
    std::vector<double> m((size_t)n * n);
    kraskov_corrmatrix(&traj, m.data(), k, true, 0);
    dump(pre + "ksg.bin", m);
    std::vector<double> r = m;
    pearsify(r.data(), n, DIM);
    write_matrix(r.data(), n, (pre + "correl.dat").c_str());
    gauss_corrmatrix(&traj, m.data());
    dump(pre + "gauss.bin", m);
    gcmi_corrmatrix(&traj, m.data(), true, 0);
    dump(pre + "gcmi.bin", m);
    te_matrix(&traj, m.data(), k, lag, true, 0);
    dump(pre + "te.bin", m);
    t_kraskov kr;
    kraskov_prepare(&traj, &kr);
    std::vector<double> w(1, kraskov_wrap(&kr, 1, 0, k));
    dump(pre + "wrap.bin", w);
    // the legacy device-facing entry on the prepared workspace
    std::fill(m.begin(), m.end(), -1.0);
    kraskov_corrmatrix_gpu(&kr, n, m.data(), k);
    dump(pre + "ksg_gpu.bin", m);
    kraskov_done(&kr);
    // input validation keeps the reference's exception and message
    t_traj one = traj;
    one.natoms = 1;
    try
    {
        kraskov_corrmatrix(&one, m.data(), k, true, 0);
        std::puts("no-throw");
    }
    catch (const std::runtime_error& e)
    {
        std::printf("throw: %s\n", e.what());
    }
    std::printf("gpu_available=%d\n", gpu_available() ? 1 : 0);
    std::printf("kraskov_gpu_probe=%d\n", kraskov_gpu_probe() ? 1 : 0);
    done_traj(&traj);
    return 0;
}
