// C++ drop-in for polysolve's MAS solver, header-only over the C ABI (include/polysolve_mas.h).
//
// Mirrors polysolve::linear::Solver (src/polysolve/linear/Solver.hpp:31-132) and MASSolver
// (src/polysolve/linear/MASSolver.hpp:35-72): Solver::create(name, precond) / create(json),
// set_parameters(json), get_info(json&), analyze_pattern(A, precond_num), factorize(A),
// solve(b, x), name(). Non-zero statuses become the reference's exception types:
// CudaOutOfMemoryError for device OOM (mas_utils/CudaUtils.cuh:33-37), std::runtime_error
// otherwise, with the "[MAS] ..." messages.
//
// Types are templates so the header needs neither Eigen nor nlohmann::json:
//   * a matrix is anything with rows(), nonZeros(), outerIndexPtr(), innerIndexPtr(), valuePtr()
//     in compressed column-major form (Eigen::SparseMatrix<double, ColMajor, int>, or CscView);
//   * a vector is anything with data() and size() (Eigen::VectorXd, std::vector<double>);
//   * a json is anything with dump() (parameters) and, for get_info, parse(string) + update()
//     (nlohmann::json), or a std::string holding JSON text.
#pragma once

#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../polysolve_mas.h"

#define POLYSOLVE_DELETE_MOVE_COPY(Base) \
    Base(Base &&) = delete;              \
    Base &operator=(Base &&) = delete;   \
    Base(const Base &) = delete;         \
    Base &operator=(const Base &) = delete;

namespace polysolve::linear
{
    namespace mas
    {
        class CudaOutOfMemoryError : public std::runtime_error
        {
        public:
            using std::runtime_error::runtime_error;
        };
    } // namespace mas

    /// Compressed column view (the layout of polysolve's StiffnessMatrix, Types.hpp:11).
    struct CscView
    {
        int n = 0;
        int nnz = 0;
        const int *outer = nullptr;
        const int *inner = nullptr;
        const double *vals = nullptr;
        int rows() const { return n; }
        int nonZeros() const { return nnz; }
        const int *outerIndexPtr() const { return outer; }
        const int *innerIndexPtr() const { return inner; }
        const double *valuePtr() const { return vals; }
    };

    enum class MASSolverStatus
    {
        Running,
        ReachRelativeTolerance,
        ReachAbsoluteTolerance,
        ReachMaxIterations,
    };

    inline std::string mas_status_to_string(MASSolverStatus stat)
    {
        switch (stat)
        {
        case MASSolverStatus::Running:
            return "Running";
        case MASSolverStatus::ReachRelativeTolerance:
            return "Reach relative tolerance";
        case MASSolverStatus::ReachAbsoluteTolerance:
            return "Reach absolute tolerance";
        case MASSolverStatus::ReachMaxIterations:
            return "Reach max iterations";
        default:
            return "Unknown";
        }
    }

    namespace detail
    {
        inline void throw_status(int rc, const char *msg)
        {
            std::string m = (msg && *msg) ? msg : ("[MAS] error " + std::to_string(rc));
            if (rc == MAS_ERR_OOM)
                throw mas::CudaOutOfMemoryError(m);
            throw std::runtime_error(m);
        }

        template <class J>
        std::string to_text(const J &j)
        {
            return j.dump();
        }
        inline std::string to_text(const std::string &s) { return s; }
        inline std::string to_text(const char *s) { return s ? s : "{}"; }
    } // namespace detail

    class Solver
    {
    public:
        virtual ~Solver()
        {
            mas_destroy(h_);
        }
        POLYSOLVE_DELETE_MOVE_COPY(Solver)

        /// Solver::create(solver, precond): only "MAS" (Solver.cpp:403-407).
        static std::unique_ptr<Solver> create(const std::string &solver, const std::string &precond)
        {
            mas_solver *h = nullptr;
            int rc = mas_create(solver.c_str(), precond.c_str(), &h);
            if (rc != MAS_OK)
                detail::throw_status(rc, mas_last_error(nullptr));
            return std::unique_ptr<Solver>(new Solver(h));
        }

        /// Solver::create(json, logger, strict) (Solver.cpp:145-167): spec validation + defaults.
        /// Enabled for json types with dump() (nlohmann::json); JSON text goes to create_from_text.
        template <class J, class Logger, class = decltype(std::declval<const J &>().dump())>
        static std::unique_ptr<Solver> create(const J &params, Logger &, bool strict_validation = true)
        {
            return create_from_text(params.dump(), strict_validation);
        }
        static std::unique_ptr<Solver> create_from_text(const std::string &params_json, bool strict = true)
        {
            mas_solver *h = nullptr;
            int rc = mas_create_json(params_json.c_str(), strict ? 1 : 0, &h);
            if (rc != MAS_OK)
                detail::throw_status(rc, mas_last_error(nullptr));
            return std::unique_ptr<Solver>(new Solver(h));
        }

        static std::vector<std::string> available_solvers() { return {"MAS"}; }
        static std::string default_solver() { return "MAS"; }

        /// MASSolver::set_parameters: reads params["MAS"], silently ignores its absence.
        template <class J>
        void set_parameters(const J &params)
        {
            check(mas_set_parameters(h_, detail::to_text(params).c_str()));
        }

        /// MASSolver::get_info as JSON text (solver_iter, solver_error, solver_status, ...).
        std::string info() const
        {
            size_t need = 0;
            mas_get_info(h_, nullptr, 0, &need);
            std::string s(need, '\0');
            mas_get_info(h_, s.data(), need, &need);
            s.resize(need ? need - 1 : 0);
            return s;
        }

        /// get_info(json&): merges the keys into `params` (nlohmann::json style).
        template <class J>
        void get_info(J &params) const
        {
            params.update(J::parse(info()));
        }
        void get_info(std::string &params) const { params = info(); }

        template <class M>
        void analyze_pattern(const M &A, const int precond_num)
        {
            check(mas_analyze_pattern(h_, (int)A.rows(), A.outerIndexPtr(), A.innerIndexPtr(), (int)A.nonZeros(),
                                      precond_num));
        }

        /// New: vertex positions for the Morton subdomain ordering (xyz per block row).
        void set_positions(const double *xyz, int nverts) { check(mas_set_positions(h_, xyz, nverts)); }

        /// New: the network of "initial_guess": "learned" (MAS_WS_PARAMS float32 values).
        void set_warm_start_model(const std::vector<float> &params)
        {
            check(mas_set_warm_start_model(h_, params.data(), (long long)params.size()));
        }
        /// New: forget the kept solutions of a sequence.
        void reset_warm_start() { check(mas_reset_warm_start(h_)); }
        /// The parameters of a .psws weight file ("PSWSMPN1", four int32 dimensions, float32s).
        static std::vector<float> load_warm_start_model(const std::string &path)
        {
            std::FILE *f = std::fopen(path.c_str(), "rb");
            if (!f)
                throw std::runtime_error("[MAS] cannot open " + path);
            char magic[8];
            int dims[4];
            std::vector<float> prm(MAS_WS_PARAMS);
            const bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PSWSMPN1", 8) == 0 &&
                            std::fread(dims, sizeof(int), 4, f) == 4 && dims[0] == MAS_WS_FEATURES &&
                            dims[1] == MAS_WS_HIDDEN && dims[2] == MAS_WS_LAYERS && dims[3] == MAS_WS_PARAMS &&
                            std::fread(prm.data(), sizeof(float), prm.size(), f) == prm.size();
            std::fclose(f);
            if (!ok)
                throw std::runtime_error("[MAS] not a warm-start weight file: " + path);
            return prm;
        }

        template <class M>
        void factorize(const M &A)
        {
            check(mas_factorize_csc(h_, (int)A.rows(), A.outerIndexPtr(), A.innerIndexPtr(), A.valuePtr(),
                                    (int)A.nonZeros()));
        }

        template <class VB, class VX>
        void solve(const VB &b, VX &x)
        {
            if ((long long)b.size() != (long long)x.size())
                throw std::runtime_error("[MAS] Size mismatch. Did you forget to call factorize?");
            check(mas_solve(h_, b.data(), x.data(), (int)b.size()));
        }

        std::string name() const { return mas_name(); }

        mas_solver *handle() const { return h_; }

    private:
        explicit Solver(mas_solver *h) : h_(h) {}
        void check(int rc) const
        {
            if (rc != MAS_OK)
                detail::throw_status(rc, mas_last_error(h_));
        }
        mas_solver *h_ = nullptr;
    };

    using MASSolver = Solver;
} // namespace polysolve::linear
