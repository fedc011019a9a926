// Drives the solver through the C++ header the way polysolve's own tests drive Solver
// (tests/test_linear_solver.cpp: TEST_CASE "all" :103-164 and "pre_factor" :241-307), on a
// matrix given as Matrix Market coordinate text (symmetric or general) on the command line.
// Prints one line per check; exits non-zero on the first failure.
//
//   mas_cpp_test A.mtx

#include <polysolve/linear/MASSolver.hpp>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

using polysolve::linear::CscView;
using polysolve::linear::Solver;

namespace
{
    struct Csc
    {
        int n = 0;
        std::vector<int> outer, inner;
        std::vector<double> vals;
        CscView view() const { return CscView{n, (int)inner.size(), outer.data(), inner.data(), vals.data()}; }
    };

    // Matrix Market reader in the spirit of the reference's loadSymmetric (test_linear_solver.cpp:25-50).
    bool load_market(const std::string &path, Csc &A)
    {
        std::ifstream in(path);
        if (!in)
            return false;
        std::string line;
        bool symmetric = false;
        while (std::getline(in, line))
        {
            if (line.rfind("%%", 0) == 0)
                symmetric = line.find("symmetric") != std::string::npos;
            if (line.empty() || line[0] == '%')
                continue;
            break;
        }
        long long M = 0, N = 0, L = 0;
        std::istringstream hdr(line);
        hdr >> M >> N >> L;
        if (M != N || M <= 0)
            return false;
        std::vector<std::vector<std::pair<int, double>>> cols(N);
        for (long long k = 0; k < L; ++k)
        {
            long long i, j;
            double v;
            in >> i >> j >> v;
            cols[j - 1].push_back({(int)(i - 1), v});
            if (symmetric && i != j)
                cols[i - 1].push_back({(int)(j - 1), v});
        }
        A.n = (int)N;
        A.outer.assign(N + 1, 0);
        for (long long j = 0; j < N; ++j)
        {
            std::sort(cols[j].begin(), cols[j].end());
            A.outer[j + 1] = A.outer[j] + (int)cols[j].size();
            for (auto &e : cols[j])
            {
                A.inner.push_back(e.first);
                A.vals.push_back(e.second);
            }
        }
        return true;
    }

    std::vector<double> matvec(const Csc &A, const std::vector<double> &x)
    {
        std::vector<double> y(A.n, 0.0);
        for (int j = 0; j < A.n; ++j)
            for (int k = A.outer[j]; k < A.outer[j + 1]; ++k)
                y[A.inner[k]] += A.vals[k] * x[j];
        return y;
    }

    double residual(const Csc &A, const std::vector<double> &x, const std::vector<double> &b)
    {
        std::vector<double> y = matvec(A, x);
        double s = 0.0;
        for (int i = 0; i < A.n; ++i)
            s += (y[i] - b[i]) * (y[i] - b[i]);
        return std::sqrt(s);
    }

    int fail(const char *what, double v)
    {
        std::printf("FAIL %s %.3e\n", what, v);
        return 1;
    }
} // namespace

int main(int argc, char **argv)
{
    if (argc < 2)
    {
        std::printf("usage: %s A.mtx\n", argv[0]);
        return 2;
    }
    Csc A;
    if (!load_market(argv[1], A))
        return fail("load", 0.0);

    // TEST_CASE("all"): rel 0, abs 1e-8, ||Ax - b|| < 1e-8.
    {
        auto solver = Solver::create("MAS", "");
        solver->set_parameters(std::string("{\"MAS\": {\"tolerance\": 1e-10}}"));
        solver->set_parameters(std::string(
            "{\"MAS\": {\"relative_tolerance\": 0.0, \"absolute_tolerance\": 1e-8, "
            "\"use_preconditioned_residual_norm\": false}}"));
        std::mt19937 eng(0);
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        std::vector<double> b(A.n), x(A.n, 0.0);
        for (double &v : b)
            v = u(eng);
        solver->analyze_pattern(A.view(), A.n);
        solver->factorize(A.view());
        solver->solve(b, x);
        if (solver->name() != "MAS")
            return fail("name", 0.0);
        std::string info;
        solver->get_info(info);
        const double err = residual(A, x, b);
        std::printf("all: err %.3e info %s\n", err, info.c_str());
        if (!(err < 1e-8))
            return fail("all", err);
    }

    // TEST_CASE("pre_factor"): 10 refactorizations with random SPD-ish values on the same pattern.
    {
        auto solver = Solver::create("MAS", "");
        solver->set_parameters(std::string(
            "{\"MAS\": {\"relative_tolerance\": 0.0, \"absolute_tolerance\": 1e-9, \"lazy_partitioning\": true}}"));
        solver->analyze_pattern(A.view(), A.n);
        std::default_random_engine eng{42};
        std::uniform_real_distribution<double> urd(0.1, 5);
        for (int round = 0; round < 10; ++round)
        {
            Csc T = A;
            // upper entries drawn in column order, mirrored to the lower triangle
            std::vector<std::vector<double>> upper(A.n);
            for (int j = 0; j < A.n; ++j)
                for (int k = A.outer[j]; k < A.outer[j + 1]; ++k)
                {
                    const int i = A.inner[k];
                    if (i == j)
                        T.vals[k] = urd(eng) * 100;
                    else if (i < j)
                        T.vals[k] = -urd(eng);
                }
            for (int j = 0; j < A.n; ++j)
                for (int k = A.outer[j]; k < A.outer[j + 1]; ++k)
                {
                    const int i = A.inner[k];
                    if (i > j)
                    {
                        // find (j, i) in column i
                        for (int q = A.outer[i]; q < A.outer[i + 1]; ++q)
                            if (A.inner[q] == j)
                                T.vals[k] = T.vals[q];
                    }
                }
            std::vector<double> b(A.n), x(A.n, 0.0);
            std::uniform_real_distribution<double> u(-1.0, 1.0);
            for (double &v : b)
                v = u(eng);
            solver->factorize(T.view());
            solver->solve(b, x);
            const double err = residual(T, x, b);
            std::printf("pre_factor %d: err %.3e\n", round, err);
            if (!(err < 1e-8))
                return fail("pre_factor", err);
        }
    }

    // Errors surface as the reference's exception types.
    {
        auto solver = Solver::create("MAS", "");
        std::vector<double> b(3, 1.0), x(3, 0.0);
        bool threw = false;
        try
        {
            solver->solve(b, x);
        }
        catch (const std::runtime_error &e)
        {
            threw = std::string(e.what()).find("Did you forget to call factorize") != std::string::npos;
        }
        if (!threw)
            return fail("solve before factorize", 0.0);
        threw = false;
        try
        {
            Solver::create("Eigen::SimplicialLDLT", "");
        }
        catch (const std::runtime_error &)
        {
            threw = true;
        }
        if (!threw)
            return fail("unknown solver", 0.0);
    }
    std::printf("OK\n");
    return 0;
}
