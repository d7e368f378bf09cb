// gmx_correlation_b200 -- standalone front end of the all-pairs path.
//
// Mirrors the options and the dispatch of the reference's GROMACS module
// (src/gmx_correlation.cpp:77-135 options, :247-355 writeOutput): GCMI
// (-gcmi) before Gaussian (-linear) before KSG, pearsify unless -mi, an
// optional transfer-entropy matrix (-te, -lag, -ote), correl.dat (-o) and
// XPM (-m) output.  GROMACS trajectory reading (src/gmx_correlation.cpp:
// 158-223) is replaced by the library's native XTC / TRR reader
// (gc_traj_read: the atoms of an index group (-n, -sel) or of an atom-number
// list (-sel "1-100 120"), frames inside -b / -e, every -skip-th, each atom's
// mean subtracted as finishAnalysis does), and the reference's own -dump
// text format (src/gmx_correlation.cpp:225-244) is read as well: a
// "natoms nframes" line, then per frame and atom one "x y z" line of
// mean-centred coordinates.  The estimators are called only through the
// drop-in C++ interface (correlation_core.h, gcmi.h, transfer_entropy.h),
// i.e. exactly what the reference front end links against.

#include "correlation_core.h"
#include "gcmi.h"
#include "gmx_corr_b200.h"
#include "transfer_entropy.h"

#include <cmath>
#include <fstream>
#include <sstream>

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
    std::string in, out = "correl.dat", xpm, ote, dump, sel, ndx;
    int         skip = 1, k = 100, nt = 0, lag = 1;
    double      tb = NAN, te_ = NAN;
    bool        linear = false, mi = false, gpu = false, gcmi = false, te = false, fit = false;
};

void usage()
{
    std::fprintf(stderr,
                 "usage: gmx_correlation_b200 -f traj.xtc|traj.trr|traj_dump.txt [-n index.ndx] [-sel group|\"1-100\"]\n"
                 "       [-b t0] [-e t1] [-o correl.dat] [-m correl.xpm] [-k 100]\n"
                 "       [-skip 1] [-linear] [-mi] [-gpu] [-nt 0] [-gcmi] [-te] [-lag 1] [-ote te.dat]\n"
                 "       [-dump out_dump.txt]\n");
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
        else if (flag(a, "-n"))
            o.ndx = next();
        else if (flag(a, "-b"))
            o.tb = std::atof(next());
        else if (flag(a, "-e"))
            o.te_ = std::atof(next());
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
        throw std::runtime_error("-f <trajectory: .xtc, .trr or -dump text> is required");
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

// 0-based atom indices of an index group (-n file, -sel name) or of an
// atom-number list such as "1-100 120" (1-based, inclusive ranges).
std::vector<int> selection(const Options& o)
{
    std::vector<int> atoms;
    if (!o.ndx.empty())
    {
        std::ifstream f(o.ndx);
        if (!f)
            throw std::runtime_error("Cannot open index file " + o.ndx);
        std::string line, group;
        bool        found = false, in_group = false;
        std::vector<std::string> names;
        while (std::getline(f, line))
        {
            line = line.substr(0, line.find(';'));
            const size_t l = line.find('['), r = line.find(']');
            if (l != std::string::npos && r != std::string::npos && r > l)
            {
                std::string nm = line.substr(l + 1, r - l - 1);
                nm.erase(0, nm.find_first_not_of(" \t"));
                nm.erase(nm.find_last_not_of(" \t") + 1);
                names.push_back(nm);
                in_group = !found && nm == o.sel;
                found    = found || in_group;
                continue;
            }
            if (!in_group)
                continue;
            std::istringstream is(line);
            long               v;
            while (is >> v)
            {
                if (v < 1)
                    throw std::runtime_error("index file " + o.ndx + ": atom number below 1");
                atoms.push_back((int)(v - 1));
            }
        }
        if (!found)
        {
            std::string all;
            for (const auto& n : names)
                all += " '" + n + "'";
            throw std::runtime_error("-sel: no group '" + o.sel + "' in " + o.ndx + " (groups:" + all + ")");
        }
        if (atoms.empty())
            throw std::runtime_error("-sel: group '" + o.sel + "' is empty");
        return atoms;
    }
    if (o.sel.empty())
        return atoms; // every atom
    std::string spec = o.sel;
    for (char& c : spec)
        if (c == ',')
            c = ' ';
    std::istringstream is(spec);
    std::string        tok;
    while (is >> tok)
    {
        const size_t dash = tok.find('-');
        char*        end  = nullptr;
        const long   a    = std::strtol(tok.c_str(), &end, 10);
        long         b    = a;
        if (dash != std::string::npos && dash > 0)
            b = std::strtol(tok.c_str() + dash + 1, &end, 10);
        if (!end || *end != 0 || a < 1 || b < a)
            throw std::runtime_error("-sel: '" + tok + "' is neither an index group (give -n) nor an atom range");
        for (long v = a; v <= b; ++v)
            atoms.push_back((int)(v - 1));
    }
    return atoms;
}

// XTC / TRR through the library reader; fills traj as finishAnalysis does.
bool read_binary(const Options& o, t_traj* traj)
{
    int fmt = 0;
    {
        FILE* f = std::fopen(o.in.c_str(), "rb");
        if (!f)
            throw std::runtime_error("Cannot open trajectory: " + o.in);
        unsigned char b[4] = {0, 0, 0, 0};
        const size_t  n    = std::fread(b, 1, 4, f);
        std::fclose(f);
        const int m = n == 4 ? (b[0] << 24 | b[1] << 16 | b[2] << 8 | b[3]) : 0;
        fmt         = m == 1995 ? GC_TRAJ_XTC : (m == 1993 ? GC_TRAJ_TRR : 0);
    }
    if (!fmt)
        return false;
    const std::vector<int> atoms = selection(o);
    gc_traj_select         s{};
    s.atoms  = atoms.empty() ? nullptr : atoms.data();
    s.natoms = (int)atoms.size();
    s.skip   = o.skip;
    s.flags  = GC_TRAJ_CENTER;
    if (!std::isnan(o.tb))
    {
        s.t_begin = o.tb;
        s.flags |= GC_TRAJ_BEGIN;
    }
    if (!std::isnan(o.te_))
    {
        s.t_end = o.te_;
        s.flags |= GC_TRAJ_END;
    }
    double* xyz = nullptr;
    int     n = 0, T = 0;
    if (gc_traj_read(o.in.c_str(), &s, &xyz, &n, &T) != GC_OK)
        throw std::runtime_error(gc_last_error());
    traj->natoms  = n;
    traj->nframes = T;
    snew(traj->x, n);
    snew(traj->xav, n);
    for (int a = 0; a < n; ++a)
    {
        snew(traj->x[a], T);
        for (int t = 0; t < T; ++t)
            for (int d = 0; d < 3; ++d)
                traj->x[a][t][d] = xyz[((size_t)a * T + t) * 3 + d];
    }
    gc_traj_free(xyz);
    return true;
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
    if (!read_binary(o, &traj))
    {
        if (!o.ndx.empty() || !o.sel.empty() || !std::isnan(o.tb) || !std::isnan(o.te_))
            throw std::runtime_error("-n, -sel, -b and -e apply to XTC / TRR input, not to a -dump file");
        read_dump(o, &traj);
    }
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
        const std::string title = (o.sel.empty() ? std::string("selection") : o.sel) + " correlation matrix";
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
