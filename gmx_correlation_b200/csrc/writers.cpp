// Output side of the path: pearsify and the two matrix writers, byte-for-byte
// compatible with lib/correlation_core.cpp:202-278 and :461-469 so existing
// consumers (bin/analyze_matrix.py read_matrix, XPM viewers) read our files
// unchanged.  The formats are the reference's file contract, hence the same
// printf conversions.

#include "gmx_corr_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>

extern "C" {

void gc_pearsify(double* mat, int n, int dim)
{
    if (!mat || n <= 0 || dim <= 0)
        return;
    const double scale = -2.0 / dim;
    const long   nn    = (long)n * n;
    for (long i = 0; i < nn; ++i)
        mat[i] = mat[i] > 0.0 ? std::sqrt(1.0 - std::exp(scale * mat[i])) : 0.0;
}

gc_status gc_write_matrix(const double* mat, int n, const char* path)
{
    if (!mat || !path || n < 0)
        return GC_ERR_INVALID;
    FILE* out = std::fopen(path, "w");
    if (!out)
        return GC_ERR_IO;
    std::fprintf(out, "%d x %d [\n", n, n);
    int ncol = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            // Column-major: the file's row i holds matrix column i.
            std::fprintf(out, "%10.6g ", mat[(size_t)j * n + i]);
            if (++ncol > 20)
            {
                ncol = 0;
                std::fputc('\n', out);
            }
        }
    std::fputs("]\n", out);
    return std::fclose(out) == 0 ? GC_OK : GC_ERR_IO;
}

gc_status gc_write_xpm(const double* mat, int n, const char* path, const char* title, const char* legend)
{
    if (!mat || !path || n < 0)
        return GC_ERR_INVALID;
    FILE* out = std::fopen(path, "w");
    if (!out)
        return GC_ERR_IO;
    double lo = 1e100, hi = -1e100;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (i != j)
            {
                const double v = mat[(size_t)j * n + i];
                lo             = std::min(lo, v);
                hi             = std::max(hi, v);
            }
    if (lo >= hi)
    {
        lo = 0.0;
        hi = 1.0;
    }
    const int levels = 80;
    std::fprintf(out, "/* XPM */\nstatic char *gmx_correlation_xpm[] = {\n");
    std::fprintf(out, "\"%d %d %d 1\",\n", n, n, levels);
    for (int l = 0; l < levels; ++l)
    {
        const int g = 255 - static_cast<int>(255.0 * l / (levels - 1));
        std::fprintf(out, "\"%c c #%02x%02x%02x\",\n", 33 + l, g, g, g);
    }
    std::fprintf(out, "/* title: %s */\n/* legend: %s */\n", title ? title : "", legend ? legend : "");
    for (int i = 0; i < n; ++i)
    {
        std::fputc('"', out);
        for (int j = 0; j < n; ++j)
        {
            const double v = mat[(size_t)j * n + i];
            int          l = static_cast<int>((v - lo) / (hi - lo) * (levels - 1));
            l              = std::clamp(l, 0, levels - 1);
            std::fputc(33 + l, out);
        }
        std::fprintf(out, "\"%s\n", i + 1 == n ? "" : ",");
    }
    std::fprintf(out, "};\n");
    return std::fclose(out) == 0 ? GC_OK : GC_ERR_IO;
}

} // extern "C"
