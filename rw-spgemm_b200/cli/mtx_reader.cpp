#include "mtx_reader.h"

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

static std::string lower(std::string s)
{
    for (char &c : s)
        c = (char)std::tolower((unsigned char)c);
    return s;
}

int read_matrix_market(const char *path, MtxCSR *out, std::string *err)
{
    FILE *f = std::fopen(path, "r");
    if (!f)
    {
        *err = std::string("cannot open ") + path;
        return -1;
    }
    char line[4096];
    if (!std::fgets(line, sizeof(line), f))
    {
        std::fclose(f);
        *err = "empty file";
        return -2;
    }
    std::string banner = lower(line);
    if (banner.rfind("%%matrixmarket", 0) != 0 || banner.find("matrix") == std::string::npos ||
        banner.find("coordinate") == std::string::npos)
    {
        std::fclose(f);
        *err = "not a Matrix Market coordinate file";
        return -2;
    }
    const bool pattern = banner.find("pattern") != std::string::npos;
    const bool complex_ = banner.find("complex") != std::string::npos;
    const bool symmetric = banner.find("symmetric") != std::string::npos &&
                           banner.find("skew-symmetric") == std::string::npos;
    const bool hermitian = banner.find("hermitian") != std::string::npos;
    long long m = 0, n = 0, nz = 0;
    while (std::fgets(line, sizeof(line), f))
    {
        if (line[0] == '%')
            continue;
        if (std::sscanf(line, "%lld %lld %lld", &m, &n, &nz) == 3)
            break;
    }
    if (m <= 0 || n <= 0 || nz < 0 || m > 2147483647LL || n > 2147483647LL)
    {
        std::fclose(f);
        *err = "bad size line";
        return -4;
    }
    std::vector<int> ri, ci;
    std::vector<double> vv;
    ri.reserve((size_t)nz);
    ci.reserve((size_t)nz);
    vv.reserve((size_t)nz);
    long long got = 0;
    while (got < nz && std::fgets(line, sizeof(line), f))
    {
        if (line[0] == '%' || line[0] == '\n')
            continue;
        char *p = line, *e;
        long long i = std::strtoll(p, &e, 10);
        p = e;
        long long j = std::strtoll(p, &e, 10);
        p = e;
        double x = 1.0;
        if (!pattern)
        {
            x = std::strtod(p, &e); // integer, real, or the real part of complex
            (void)complex_;
        }
        if (i < 1 || i > m || j < 1 || j > n)
        {
            std::fclose(f);
            *err = "entry out of range";
            return -5;
        }
        ri.push_back((int)(i - 1));
        ci.push_back((int)(j - 1));
        vv.push_back(x);
        got++;
    }
    std::fclose(f);
    if (got != nz)
    {
        *err = "file shorter than its size line";
        return -6;
    }
    const bool mirror = symmetric || hermitian;
    std::vector<long long> cnt((size_t)m + 1, 0);
    for (long long q = 0; q < nz; q++)
    {
        cnt[ri[q] + 1]++;
        if (mirror && ri[q] != ci[q])
            cnt[ci[q] + 1]++;
    }
    for (long long r = 0; r < m; r++)
        cnt[r + 1] += cnt[r];
    if (cnt[m] > 2147483647LL)
    {
        *err = "more than 2^31-1 nonzeros";
        return -7;
    }
    out->m = (int)m;
    out->n = (int)n;
    out->nnz = (int)cnt[m];
    out->isSymmetric = mirror ? 1 : 0;
    out->rowptr.assign(cnt.begin(), cnt.end());
    out->colidx.resize((size_t)out->nnz);
    out->val.resize((size_t)out->nnz);
    std::vector<long long> fill(cnt.begin(), cnt.end() - 1);
    // same insertion order as the reference reader: file order, mirrored
    // entry right after its original
    for (long long q = 0; q < nz; q++)
    {
        long long o = fill[ri[q]]++;
        out->colidx[o] = ci[q];
        out->val[o] = vv[q];
        if (mirror && ri[q] != ci[q])
        {
            o = fill[ci[q]]++;
            out->colidx[o] = ri[q];
            out->val[o] = vv[q];
        }
    }
    return 0;
}

long long canonicalize_rows(int m, int *rowptr, int *colidx, double *val)
{
    std::vector<int> idx;
    std::vector<int> ctmp;
    std::vector<double> vtmp;
    long long w = 0; // write position: rows are compacted as duplicates go
    for (int r = 0; r < m; r++)
    {
        const int s = rowptr[r], e = rowptr[r + 1];
        idx.resize((size_t)(e - s));
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return colidx[s + a] < colidx[s + b]; });
        ctmp.assign(colidx + s, colidx + e);
        vtmp.assign(val + s, val + e);
        rowptr[r] = (int)w;
        for (int q = 0; q < e - s; q++)
        {
            const int c = ctmp[idx[q]];
            if (q > 0 && c == colidx[w - 1])
                val[w - 1] += vtmp[idx[q]];
            else
            {
                colidx[w] = c;
                val[w] = vtmp[idx[q]];
                w++;
            }
        }
    }
    const long long removed = (long long)rowptr[m] - w;
    rowptr[m] = (int)w;
    return removed;
}
