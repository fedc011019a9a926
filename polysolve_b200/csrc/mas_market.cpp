// Matrix Market files for A and b: the format polysolve's tests read with Eigen's loadMarket /
// loadMarketVector (tests/test_linear_solver.cpp:25-50, :211-213), so real systems exported by
// polyfem can replace the synthetic ones.
//
// Read: "%%MatrixMarket matrix coordinate|array real|integer|pattern general|symmetric".
// Coordinate entries are 1-based; duplicates are summed and a symmetric file (lower or upper
// triangle) is expanded to the full matrix, as Eigen's loader does. The result is CSC with sorted
// row indices (polysolve's StiffnessMatrix layout). Array files are dense column-major (a vector
// is an n x 1 array). Write: coordinate real general (or the lower triangle with "symmetric") and
// array real general for vectors, with 17 significant digits (round-trips FP64 exactly).

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/polysolve_mas.h"

namespace
{
    struct MarketError
    {
        int code;
        std::string what;
    };

    thread_local std::string g_market_error;

    struct Cursor
    {
        const char *p, *end;
        long long line = 1;

        void skip_blank()
        {
            while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n'))
            {
                if (*p == '\n')
                    ++line;
                ++p;
            }
        }
        [[noreturn]] void fail(const std::string &w) const
        {
            throw MarketError{MAS_ERR_INVALID, "[MAS] Matrix Market line " + std::to_string(line) + ": " + w};
        }
        long long integer()
        {
            skip_blank();
            long long v = 0;
            auto r = std::from_chars(p, end, v);
            if (r.ec != std::errc())
                fail("expected an integer");
            p = r.ptr;
            return v;
        }
        double real()
        {
            skip_blank();
            double v = 0.0;
            const char *q = p;
            if (q < end && *q == '+')
                ++q;
            auto r = std::from_chars(q, end, v);
            if (r.ec != std::errc())
                fail("expected a number");
            p = r.ptr;
            return v;
        }
    };

    std::string lower(std::string s)
    {
        for (char &c : s)
            c = (char)std::tolower((unsigned char)c);
        return s;
    }
} // namespace

struct mas_market
{
    int rows = 0, cols = 0;
    bool dense = false;
    std::vector<int> outer, inner;   // CSC (coordinate files)
    std::vector<double> vals;        // CSC values, or the dense column-major array
};

namespace
{
    void parse(mas_market &m, const std::string &text)
    {
        Cursor c{text.data(), text.data() + text.size()};
        // Header line.
        const size_t eol = text.find('\n');
        std::istringstream hs(lower(text.substr(0, eol)));
        std::string banner, object, format, field, symmetry;
        hs >> banner >> object >> format >> field >> symmetry;
        if (banner != "%%matrixmarket" || object != "matrix")
            c.fail("not a Matrix Market matrix file");
        if (format != "coordinate" && format != "array")
            c.fail("format must be coordinate or array");
        if (field != "real" && field != "integer" && field != "double" && field != "pattern")
            c.fail("field must be real, integer or pattern (complex is not supported)");
        if (symmetry != "general" && symmetry != "symmetric")
            c.fail("symmetry must be general or symmetric");
        const bool sym = symmetry == "symmetric";
        const bool pattern = field == "pattern";
        if (format == "array" && pattern)
            c.fail("pattern arrays are not valid");
        // Skip the header and comment lines.
        while (c.p < c.end)
        {
            c.skip_blank();
            if (c.p < c.end && *c.p == '%')
            {
                while (c.p < c.end && *c.p != '\n')
                    ++c.p;
                continue;
            }
            break;
        }
        const long long rows = c.integer(), cols = c.integer();
        if (rows < 0 || cols < 0 || rows > 2147483647LL || cols > 2147483647LL)
            c.fail("invalid size");
        if (sym && rows != cols)
            c.fail("a symmetric matrix must be square");
        m.rows = (int)rows;
        m.cols = (int)cols;
        if (format == "array")
        {
            m.dense = true;
            m.vals.assign((size_t)rows * (size_t)cols, 0.0);
            for (long long j = 0; j < cols; ++j)
                for (long long i = sym ? j : 0; i < rows; ++i)
                {
                    const double v = c.real();
                    m.vals[(size_t)j * rows + i] = v;
                    if (sym && i != j)
                        m.vals[(size_t)i * rows + j] = v;
                }
            return;
        }
        const long long entries = c.integer();
        if (entries < 0)
            c.fail("invalid entry count");
        std::vector<int> ri, ci;
        std::vector<double> vv;
        const size_t cap = (size_t)entries * (sym ? 2 : 1);
        ri.reserve(cap);
        ci.reserve(cap);
        vv.reserve(cap);
        for (long long e = 0; e < entries; ++e)
        {
            const long long i = c.integer(), j = c.integer();
            const double v = pattern ? 1.0 : c.real();
            if (i < 1 || i > rows || j < 1 || j > cols)
                c.fail("entry index out of range");
            ri.push_back((int)(i - 1));
            ci.push_back((int)(j - 1));
            vv.push_back(v);
            if (sym && i != j)
            {
                ri.push_back((int)(j - 1));
                ci.push_back((int)(i - 1));
                vv.push_back(v);
            }
        }
        if (vv.size() > 2147483647ULL)
            throw MarketError{MAS_ERR_INVALID, "[MAS] A is too large. Non-zero number exceeding int32 max."};
        // CSC: bucket by column, sort rows within a column, sum duplicates.
        std::vector<long long> start((size_t)cols + 1, 0);
        for (int j : ci)
            ++start[(size_t)j + 1];
        for (size_t j = 0; j < (size_t)cols; ++j)
            start[j + 1] += start[j];
        std::vector<std::pair<int, double>> tmp(vv.size());
        {
            std::vector<long long> fill(start.begin(), start.end() - 1);
            for (size_t k = 0; k < vv.size(); ++k)
                tmp[(size_t)fill[(size_t)ci[k]]++] = {ri[k], vv[k]};
        }
        m.outer.assign((size_t)cols + 1, 0);
        m.inner.clear();
        m.vals.clear();
        m.inner.reserve(vv.size());
        m.vals.reserve(vv.size());
        for (size_t j = 0; j < (size_t)cols; ++j)
        {
            auto b = tmp.begin() + start[j], e = tmp.begin() + start[j + 1];
            std::stable_sort(b, e, [](const auto &a, const auto &bb) { return a.first < bb.first; });
            for (auto it = b; it != e; ++it)
            {
                if (!m.inner.empty() && (long long)m.inner.size() > m.outer[j] && m.inner.back() == it->first)
                    m.vals.back() += it->second;
                else
                {
                    m.inner.push_back(it->first);
                    m.vals.push_back(it->second);
                }
            }
            m.outer[j + 1] = (int)m.inner.size();
        }
    }

    template <class F>
    int market_guard(F &&f)
    {
        try
        {
            f();
            return MAS_OK;
        }
        catch (const MarketError &e)
        {
            g_market_error = e.what;
            return e.code;
        }
        catch (const std::bad_alloc &)
        {
            g_market_error = "[MAS] out of host memory reading a Matrix Market file";
            return MAS_ERR_OOM;
        }
        catch (const std::exception &e)
        {
            g_market_error = std::string("[MAS] ") + e.what();
            return MAS_ERR_INVALID;
        }
    }

    void write_double(std::FILE *f, double v)
    {
        char buf[40];
        std::snprintf(buf, sizeof(buf), "%.17g", v);
        std::fputs(buf, f);
    }
} // namespace

extern "C" int mas_market_load(const char *path, mas_market **out)
{
    if (!path || !out)
        return MAS_ERR_INVALID;
    *out = nullptr;
    return market_guard([&] {
        std::ifstream in(path, std::ios::binary);
        if (!in)
            throw MarketError{MAS_ERR_INVALID, std::string("[MAS] cannot open ") + path};
        std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        auto m = std::make_unique<mas_market>();
        parse(*m, text);
        *out = m.release();
    });
}

extern "C" int mas_market_dims(const mas_market *m, int *rows, int *cols, long long *nnz, int *dense)
{
    if (!m)
        return MAS_ERR_INVALID;
    if (rows)
        *rows = m->rows;
    if (cols)
        *cols = m->cols;
    if (nnz)
        *nnz = m->dense ? (long long)m->vals.size() : (long long)m->inner.size();
    if (dense)
        *dense = m->dense ? 1 : 0;
    return MAS_OK;
}

extern "C" int mas_market_copy_csc(const mas_market *m, int *outer, int *inner, double *vals)
{
    if (!m || m->dense || !outer || (!m->inner.empty() && (!inner || !vals)))
        return MAS_ERR_INVALID;
    std::memcpy(outer, m->outer.data(), sizeof(int) * m->outer.size());
    if (!m->inner.empty())
    {
        std::memcpy(inner, m->inner.data(), sizeof(int) * m->inner.size());
        std::memcpy(vals, m->vals.data(), sizeof(double) * m->vals.size());
    }
    return MAS_OK;
}

extern "C" int mas_market_copy_dense(const mas_market *m, double *out, long long count)
{
    if (!m || !m->dense || count != (long long)m->vals.size() || (count > 0 && !out))
        return MAS_ERR_INVALID;
    if (count > 0)
        std::memcpy(out, m->vals.data(), sizeof(double) * (size_t)count);
    return MAS_OK;
}

extern "C" void mas_market_free(mas_market *m) { delete m; }

extern "C" const char *mas_market_last_error(void) { return g_market_error.c_str(); }

extern "C" int mas_market_write_csc(const char *path, int n, const int *outer, const int *inner, const double *vals,
                                    int symmetric)
{
    if (!path || n < 0 || !outer || (outer[n] > 0 && (!inner || !vals)))
        return MAS_ERR_INVALID;
    return market_guard([&] {
        long long count = 0;
        for (int j = 0; j < n; ++j)
            for (int k = outer[j]; k < outer[j + 1]; ++k)
            {
                if (inner[k] < 0 || inner[k] >= n)
                    throw MarketError{MAS_ERR_INVALID, "[MAS] write: row index out of range"};
                if (!symmetric || inner[k] >= j)
                    ++count;
            }
        std::FILE *f = std::fopen(path, "wb");
        if (!f)
            throw MarketError{MAS_ERR_INVALID, std::string("[MAS] cannot write ") + path};
        std::fprintf(f, "%%%%MatrixMarket matrix coordinate real %s\n%d %d %lld\n", symmetric ? "symmetric" : "general",
                     n, n, count);
        for (int j = 0; j < n; ++j)
            for (int k = outer[j]; k < outer[j + 1]; ++k)
                if (!symmetric || inner[k] >= j)
                {
                    std::fprintf(f, "%d %d ", inner[k] + 1, j + 1);
                    write_double(f, vals[k]);
                    std::fputc('\n', f);
                }
        if (std::fclose(f) != 0)
            throw MarketError{MAS_ERR_INVALID, std::string("[MAS] write failed: ") + path};
    });
}

extern "C" int mas_market_write_vector(const char *path, const double *x, long long n)
{
    if (!path || n < 0 || (n > 0 && !x) || n > 2147483647LL)
        return MAS_ERR_INVALID;
    return market_guard([&] {
        std::FILE *f = std::fopen(path, "wb");
        if (!f)
            throw MarketError{MAS_ERR_INVALID, std::string("[MAS] cannot write ") + path};
        std::fprintf(f, "%%%%MatrixMarket matrix array real general\n%lld 1\n", n);
        for (long long i = 0; i < n; ++i)
        {
            write_double(f, x[i]);
            std::fputc('\n', f);
        }
        if (std::fclose(f) != 0)
            throw MarketError{MAS_ERR_INVALID, std::string("[MAS] write failed: ") + path};
    });
}
