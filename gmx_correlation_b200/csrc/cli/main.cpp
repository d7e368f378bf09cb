// gmx_correlation_b200 -- standalone front end of the all-pairs path.
//
// Mirrors the options and the dispatch of the reference's GROMACS module
// (src/gmx_correlation.cpp:77-135 options, :247-355 writeOutput): GCMI
// (-gcmi) before Gaussian (-linear) before KSG, pearsify unless -mi, an
// optional transfer-entropy matrix (-te, -lag, -ote), correl.dat (-o) and
// XPM (-m) output.  GROMACS trajectory reading is replaced by the
// reference's own -dump text format (src/gmx_correlation.cpp:225-244):
// a "natoms nframes" line, then per frame and atom one "x y z" line of
// mean-centred coordinates.  It calls only the drop-in C++ interface
// (correlation_core.h, gcmi.h, transfer_entropy.h), i.e. exactly what the
// reference front end links against.

#include "correlation_core.h"
#include "gcmi.h"
#include "transfer_entropy.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

struct Options
{
    std::string in, out = "correl.dat", xpm, ote, dump, sel = "selection";
    int         skip = 1, k = 100, nt = 0, lag = 1;
    bool        linear = false, mi = false, gpu = false, gcmi = false, te = false, fit = false;
};

void usage()
{
    std::fprintf(stderr,
                 "usage: gmx_correlation_b200 -f traj_dump.txt [-o correl.dat] [-m correl.xpm] [-k 100]\n"
                 "       [-skip 1] [-linear] [-mi] [-gpu] [-nt 0] [-gcmi] [-te] [-lag 1] [-ote te.dat]\n"
                 "       [-dump out_dump.txt] [-sel name]\n");
}

bool flag(const char* a, const char* name) { return std::strcmp(a, name) == 0; }

Options parse(int argc, char** argv)
{
    Options o;
    for (int i = 1; i < argc; ++i)
    {
        const char* a    = argv[i];
        auto        next = [&]() -> const char* {
            if (i + 1 >= argc)
                throw std::runtime_error(std::string("missing value after ") + a);
            return argv[++i];
        };
        if (flag(a, "-f"))
            o.in = next();
        else if (flag(a, "-o"))
            o.out = next();
        else if (flag(a, "-m"))
            o.xpm = next();
        else if (flag(a, "-k"))
            o.k = std::atoi(next());
        else if (flag(a, "-skip"))
            o.skip = std::atoi(next());
        else if (flag(a, "-nt"))
            o.nt = std::atoi(next());
        else if (flag(a, "-lag"))
            o.lag = std::atoi(next());
        else if (flag(a, "-ote"))
            o.ote = next();
        else if (flag(a, "-dump"))
            o.dump = next();
        else if (flag(a, "-sel"))
            o.sel = next();
        else if (flag(a, "-linear"))
            o.linear = true;
        else if (flag(a, "-mi"))
            o.mi = true;
        else if (flag(a, "-gpu"))
            o.gpu = true;
        else if (flag(a, "-gcmi"))
            o.gcmi = true;
        else if (flag(a, "-te"))
            o.te = true;
        else if (flag(a, "-fit"))
            o.fit = true;
        else if (flag(a, "-h") || flag(a, "--help"))
        {
            usage();
            std::exit(0);
        }
        else
            throw std::runtime_error(std::string("unknown option ") + a);
    }
    if (o.in.empty())
        throw std::runtime_error("-f <trajectory dump> is required");
    // initAnalysis checks (src/gmx_correlation.cpp:139-155)
    if (o.skip < 1)
        throw std::runtime_error("The -skip value must be at least 1.");
    if (o.k < 1)
        throw std::runtime_error("The -k value must be at least 1.");
    if (o.fit)
        throw std::runtime_error("This build does not perform fitting internally. Pre-fit the trajectory with "
                                 "gmx trjconv -fit and rerun without -fit.");
    return o;
}

// Reads the -dump format; keeps every skip-th frame and, when frames were
// skipped, mean-centres the kept frames again (the reference centres after
// skipping, src/gmx_correlation.cpp:158-223).
void read_dump(const Options& o, t_traj* traj)
{
    FILE* f = std::fopen(o.in.c_str(), "r");
    if (!f)
        throw std::runtime_error("Cannot open trajectory dump: " + o.in);
    int n = 0, T = 0;
    if (std::fscanf(f, "%d %d", &n, &T) != 2 || n < 1 || T < 1)
    {
        std::fclose(f);
        throw std::runtime_error("malformed dump header in " + o.in);
    }
    const int Tk = (T + o.skip - 1) / o.skip;
    std::vector<double> xyz((size_t)n * Tk * 3);
    for (int fr = 0, kept = 0; fr < T; ++fr)
        for (int a = 0; a < n; ++a)
        {
            double v[3];
            if (std::fscanf(f, "%lf %lf %lf", &v[0], &v[1], &v[2]) != 3)
            {
                std::fclose(f);
                throw std::runtime_error("truncated dump file " + o.in);
            }
            if (fr % o.skip == 0)
            {
                const int kk = fr / o.skip;
                for (int d = 0; d < 3; ++d)
                    xyz[((size_t)a * Tk + kk) * 3 + d] = v[d];
                (void)kept;
            }
        }
    std::fclose(f);
    traj->natoms  = n;
    traj->nframes = Tk;
    snew(traj->x, n);
    snew(traj->xav, n);
    for (int a = 0; a < n; ++a)
    {
        snew(traj->x[a], Tk);
        if (o.skip > 1)
        {
            for (int fr = 0; fr < Tk; ++fr)
                for (int d = 0; d < 3; ++d)
                    traj->xav[a][d] += xyz[((size_t)a * Tk + fr) * 3 + d];
            for (int d = 0; d < 3; ++d)
                traj->xav[a][d] /= Tk;
        }
        for (int fr = 0; fr < Tk; ++fr)
            for (int d = 0; d < 3; ++d)
                traj->x[a][fr][d] = xyz[((size_t)a * Tk + fr) * 3 + d] - traj->xav[a][d];
    }
}

void write_dump(const std::string& path, const t_traj& t)
{
    FILE* dp = std::fopen(path.c_str(), "w");
    if (!dp)
        throw std::runtime_error("Cannot open dump file: " + path);
    std::fprintf(dp, "%d %d\n", t.natoms, t.nframes);
    for (int fr = 0; fr < t.nframes; ++fr)
        for (int a = 0; a < t.natoms; ++a)
            std::fprintf(dp, "%.10g %.10g %.10g\n", t.x[a][fr][0], t.x[a][fr][1], t.x[a][fr][2]);
    std::fclose(dp);
}

int run(const Options& o)
{
    t_traj traj;
    read_dump(o, &traj);
    if (o.k >= traj.nframes)
        throw std::runtime_error("The -k value must be smaller than the number of analyzed frames.");
    if (!o.dump.empty())
        write_dump(o.dump, traj);
    const int           n = traj.natoms, T = traj.nframes;
    std::vector<double> result((size_t)n * n, 1.0);
    using Clock = std::chrono::steady_clock;
    if (o.gcmi)
    {
        std::fprintf(stderr, "\nComputing GCMI correlation matrix (%d atoms, %d frames) on GPU...\n", n, T);
        const auto t0 = Clock::now();
        gcmi_corrmatrix(&traj, result.data(), true, o.nt);
        std::fprintf(stderr, "GCMI matrix done in %.2f s\n",
                     std::chrono::duration<double>(Clock::now() - t0).count());
    }
    else if (o.linear)
    {
        std::fprintf(stderr, "\nComputing Gaussian correlation matrix (%d atoms, %d frames)...\n", n, T);
        const auto t0 = Clock::now();
        gauss_corrmatrix(&traj, result.data());
        std::fprintf(stderr, "Gaussian matrix done in %.2f s\n",
                     std::chrono::duration<double>(Clock::now() - t0).count());
    }
    else
    {
        std::fprintf(stderr, "\nComputing Kraskov correlation matrix (%d atoms, %d frames, k=%d) on GPU...\n", n,
                     T, o.k);
        const auto t0 = Clock::now();
        kraskov_corrmatrix(&traj, result.data(), o.k, true, o.nt);
        std::fprintf(stderr, "Kraskov matrix done in %.2f s\n",
                     std::chrono::duration<double>(Clock::now() - t0).count());
    }
    if (!o.mi)
    {
        if (o.gcmi)
            std::fprintf(stderr, "NOTE: Applying Lange-Grubmuller r(MI) conversion to GCMI output.\n"
                                 "      This transform was validated for KSG MI, not GCMI.\n"
                                 "      Use -mi to write raw MI (nats) if in doubt.\n");
        pearsify(result.data(), n, DIM);
    }
    if (o.te)
    {
        std::vector<double> te((size_t)n * n, 0.0);
        std::fprintf(stderr, "\nComputing transfer entropy matrix (%d atoms, %d frames, k=%d, lag=%d) on GPU...\n",
                     n, T, o.k, o.lag);
        const auto t0 = Clock::now();
        te_matrix(&traj, te.data(), o.k, o.lag, true, o.nt);
        std::fprintf(stderr, "Transfer entropy matrix done in %.2f s\n",
                     std::chrono::duration<double>(Clock::now() - t0).count());
        if (!o.ote.empty())
        {
            std::fprintf(stderr, "Writing TE matrix to %s\n", o.ote.c_str());
            write_matrix(te.data(), n, o.ote.c_str());
        }
        else
            std::fprintf(stderr, "Note: use -ote <file> to save the transfer entropy matrix.\n");
    }
    std::fprintf(stderr, "Writing output to %s\n", o.out.c_str());
    write_matrix(result.data(), n, o.out.c_str());
    if (!o.xpm.empty())
    {
        const std::string title = o.sel + " correlation matrix";
        write_xpm_matrix(result.data(), n, o.xpm.c_str(), title.c_str(), o.mi ? "MI (bits)" : "r(MI)");
        std::fprintf(stderr, "Writing XPM to %s\n", o.xpm.c_str());
    }
    done_traj(&traj);
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    try
    {
        return run(parse(argc, argv));
    }
    catch (const std::exception& e)
    {
        std::fprintf(stderr, "Error: %s\n", e.what());
        usage();
        return 1;
    }
}
