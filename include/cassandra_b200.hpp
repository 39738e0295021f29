// cassandra_b200.hpp — header-only C++ drop-in for the reference's fitting
// API, implemented over the C ABI in cassandra_b200.h.  The names, argument
// meaning and error behaviour follow the reference:
//
//   Vector                        Math/Vector.h:5        (std::vector<float>)
//   MatrixCSR                     Math/MatrixCSR.h:11-26
//   operator*(MatrixCSR, Vector)  Math/MatrixCSR.h:32    y = A x
//   operator*(Vector, MatrixCSR)  Math/MatrixCSR.h:33    x = A' y
//   JacobiPreconditionerOfATA     Math/MatrixCSR.h:30
//   transposed(), A' * A proxy    Math/MatrixProxy.h:34-77
//   DiagonalPreconditioner        Math/Solver.h:25-38
//   PCG, CG, LSQR, LSMR           Math/Solver.h:40-287   Iterate/Residuum/Error/X
//   GroupIndexer                  Pattern/Indexer.h:29-40
//   FitWeights                    PatternFit/PatternFit.cpp:7-39
//
// Dimension errors throw std::runtime_error("Size mismatch."), as the
// reference does; other failures throw std::runtime_error with the library's
// message.  All arithmetic runs on the GPU: a MatrixCSR keeps a host copy of
// its indices (Row(i) is writable as in the reference) and uploads it once,
// on first use, to a device-resident CSR with its sorted transposed copy.
// Vectors stay std::vector<float> at the API; solvers keep their state on
// the device in FP64 and return float vectors from X() and Error().
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "cassandra_b200.h"

namespace cassandra_b200 {

using Vector = std::vector<float>;

inline void check(cas_status s)
{
    if (s == CAS_OK) return;
    if (s == CAS_ERR_SIZE_MISMATCH) throw std::runtime_error("Size mismatch.");
    char buf[512];
    cas_last_error(buf, sizeof buf);
    throw std::runtime_error(std::string(cas_status_name(s)) + ": " + buf);
}

namespace detail {
template <typename T>
struct DeviceBuffer {
    T* p = nullptr;
    size_t n = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t count) : n(count)
    {
        if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess)
            throw std::runtime_error("cudaMalloc failed");
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; }
    ~DeviceBuffer() { cudaFree(p); }
    void upload(const T* h, size_t count)
    {
        if (count && cudaMemcpy(p, h, sizeof(T) * count, cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("cudaMemcpy failed");
    }
    void download(T* h, size_t count) const
    {
        if (count && cudaMemcpy(h, p, sizeof(T) * count, cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("cudaMemcpy failed");
    }
};

inline DeviceBuffer<double> to_device_f64(const Vector& v)
{
    std::vector<double> d(v.begin(), v.end());
    DeviceBuffer<double> b(d.size());
    b.upload(d.data(), d.size());
    return b;
}

inline Vector to_host_f32(const DeviceBuffer<double>& b, size_t n)
{
    std::vector<double> d(n);
    b.download(d.data(), n);
    return Vector(d.begin(), d.end());
}
}  // namespace detail

// Vector algebra of Math/Vector.h:7-31 on host vectors (the solvers keep
// their own vectors on the device; these serve callers' host-side code).
namespace vector_ops {
inline void same_size(const Vector& a, const Vector& b)
{
    if (a.size() != b.size()) throw std::runtime_error("Size mismatch");
}
}  // namespace vector_ops
inline void operator+=(Vector& l, const Vector& o)
{
    vector_ops::same_size(l, o);
    for (size_t i = 0; i < l.size(); i++) l[i] += o[i];
}
inline void operator-=(Vector& l, const Vector& o)
{
    vector_ops::same_size(l, o);
    for (size_t i = 0; i < l.size(); i++) l[i] -= o[i];
}
inline void operator*=(Vector& l, float f)
{
    for (float& v : l) v *= f;
}
inline void operator/=(Vector& l, float f)
{
    for (float& v : l) v /= f;
}
inline Vector operator+(Vector l, const Vector& r)
{
    l += r;
    return l;
}
inline Vector operator-(Vector l, const Vector& r)
{
    l -= r;
    return l;
}
inline Vector operator*(Vector v, float f)
{
    v *= f;
    return v;
}
inline Vector operator*(float f, Vector v)
{
    v *= f;
    return v;
}
inline Vector operator/(Vector v, float f)
{
    v /= f;
    return v;
}
inline Vector elementwise_multiplication(Vector l, const Vector& o)
{
    vector_ops::same_size(l, o);
    for (size_t i = 0; i < l.size(); i++) l[i] *= o[i];
    return l;
}
inline Vector elementwise_division(Vector l, const Vector& o)
{
    vector_ops::same_size(l, o);
    for (size_t i = 0; i < l.size(); i++) l[i] /= o[i];
    return l;
}
inline Vector inv(Vector v)
{
    for (float& x : v) x = 1.0f / x;
    return v;
}
inline float dot(const Vector& l, const Vector& r)
{
    vector_ops::same_size(l, r);
    double s = 0;
    for (size_t i = 0; i < l.size(); i++) s += double(l[i]) * r[i];
    return static_cast<float>(s);
}
inline float norm(const Vector& x) { return std::sqrt(dot(x, x)); }
inline float L2_norm(const Vector& x) { return norm(x); }
inline float L1_norm(const Vector& x)
{
    double s = 0;
    for (float v : x) s += std::fabs(v);
    return static_cast<float>(s);
}
inline float sum(const Vector& x)
{
    double s = 0;
    for (float v : x) s += v;
    return static_cast<float>(s);
}

// Compressed sparse row matrix with a fixed number of entries per row and
// implicit 1.0 values; duplicate column indices in a row add up.
class MatrixCSR {
    std::size_t elements_per_row;
    std::size_t cols;
    std::vector<uint32_t> col_indices;
    mutable cas_csr* dev = nullptr;

public:
    MatrixCSR(std::size_t elements_per_row, std::size_t rows, std::size_t cols)
        : elements_per_row(elements_per_row), cols(cols), col_indices(rows * elements_per_row)
    {
    }
    MatrixCSR(const MatrixCSR& o) : elements_per_row(o.elements_per_row), cols(o.cols), col_indices(o.col_indices) {}
    MatrixCSR(MatrixCSR&& o) noexcept
        : elements_per_row(o.elements_per_row), cols(o.cols), col_indices(std::move(o.col_indices)), dev(o.dev)
    {
        o.dev = nullptr;
    }
    ~MatrixCSR() { cas_csr_destroy(dev); }

    std::size_t Rows() const noexcept { return elements_per_row ? col_indices.size() / elements_per_row : 0; }
    std::size_t Cols() const noexcept { return cols; }
    std::size_t ElementsPerRow() const noexcept { return elements_per_row; }

    // Writable row access invalidates the device copy.
    std::span<uint32_t> Row(std::size_t i) noexcept
    {
        invalidate();
        return {col_indices.data() + i * elements_per_row, elements_per_row};
    }
    std::span<const uint32_t> Row(std::size_t i) const noexcept
    {
        return {col_indices.data() + i * elements_per_row, elements_per_row};
    }

    void invalidate() noexcept
    {
        cas_csr_destroy(dev);
        dev = nullptr;
    }

    // Device-resident CSR (built on first use).
    const cas_csr* device() const
    {
        if (!dev) {
            detail::DeviceBuffer<uint32_t> idx(col_indices.size());
            idx.upload(col_indices.data(), col_indices.size());
            check(cas_csr_from_indices(idx.p, static_cast<int>(elements_per_row), static_cast<int64_t>(Rows()),
                                       static_cast<int64_t>(cols), nullptr, &dev));
        }
        return dev;
    }
};

// y = A x (Math/MatrixCSR.cpp:49-65).
inline Vector operator*(const MatrixCSR& a, const Vector& x)
{
    if (x.size() != a.Cols()) throw std::runtime_error("Size mismatch.");
    detail::DeviceBuffer<float> dx(x.size()), dy(a.Rows());
    dx.upload(x.data(), x.size());
    check(cas_spmv(a.device(), CAS_F32, dx.p, dy.p, nullptr));
    Vector y(a.Rows());
    dy.download(y.data(), y.size());
    return y;
}

// x = A' y (Math/MatrixCSR.cpp:67-87).
inline Vector operator*(const Vector& y, const MatrixCSR& a)
{
    if (y.size() != a.Rows()) throw std::runtime_error("Size mismatch.");
    detail::DeviceBuffer<float> dy(y.size()), dx(a.Cols());
    dy.upload(y.data(), y.size());
    check(cas_spmv_t(a.device(), CAS_F32, dy.p, dx.p, nullptr));
    Vector x(a.Cols());
    dx.download(x.data(), x.size());
    return x;
}

// 1 / diag(A'A) (Math/MatrixCSR.cpp:21-47).
inline Vector JacobiPreconditionerOfATA(const MatrixCSR& a)
{
    detail::DeviceBuffer<float> d(a.Cols());
    check(cas_jacobi(a.device(), CAS_F32, d.p, nullptr));
    Vector out(a.Cols());
    d.download(out.data(), out.size());
    return out;
}

// Lazy transposed matrix and product proxies (Math/MatrixProxy.h:9-77): they
// only record the structure, so PCG(transposed(A) * A, ...) never forms A'A.
template <typename T>
struct TransposedMatrix {
    const T& m;
    explicit TransposedMatrix(const T& m) noexcept : m(m) {}
    std::size_t Rows() const noexcept { return m.Cols(); }
    std::size_t Cols() const noexcept { return m.Rows(); }
};

template <typename T>
auto transposed(const T& m)
{
    return TransposedMatrix<T>(m);
}

template <typename T>
Vector operator*(const TransposedMatrix<T>& t, const Vector& x)
{
    return x * t.m;
}

template <typename T>
Vector operator*(const Vector& x, const TransposedMatrix<T>& t)
{
    return t.m * x;
}

template <typename L, typename R>
struct TwoMatrix {
    const L& l;
    const R& r;
    TwoMatrix(const L& l, const R& r) : l(l), r(r)
    {
        if (l.Cols() != r.Rows()) throw std::runtime_error("Size mismatch.");
    }
    std::size_t Rows() const noexcept { return l.Rows(); }
    std::size_t Cols() const noexcept { return r.Cols(); }
};

inline TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR> operator*(const TransposedMatrix<MatrixCSR>& l,
                                                                   const MatrixCSR& r)
{
    return {l, r};
}

template <typename L, typename R>
Vector operator*(const TwoMatrix<L, R>& m, const Vector& x)
{
    return m.l * (m.r * x);
}

class Preconditioner {
public:
    virtual ~Preconditioner() = default;
    virtual Vector apply(const Vector&) const = 0;
    virtual Vector revert(const Vector&) const = 0;
};

// Math/Solver.h:25-38: entries that are not normal become 1.
class DiagonalPreconditioner : public Preconditioner {
public:
    Vector d;
    explicit DiagonalPreconditioner(Vector dd) : d(std::move(dd))
    {
        for (float& v : d)
            if (!std::isnormal(v)) v = 1;
    }
    Vector apply(const Vector& x) const override
    {
        if (x.size() != d.size()) throw std::runtime_error("Size mismatch");
        Vector r(x.size());
        for (size_t i = 0; i < x.size(); i++) r[i] = d[i] * x[i];
        return r;
    }
    Vector revert(const Vector& x) const override
    {
        if (x.size() != d.size()) throw std::runtime_error("Size mismatch");
        Vector r(x.size());
        for (size_t i = 0; i < x.size(); i++) r[i] = d[i] / x[i];
        return r;
    }
};

class IterativeSolver {
public:
    virtual ~IterativeSolver() = default;
    virtual void Iterate(int n = 1) = 0;
    virtual float Residuum() const = 0;
    virtual Vector Error() const = 0;
    virtual Vector X() const = 0;
};

namespace detail {
// Device solver state: the recurrences of Math/Solver.h run in FP64 on the
// device; rhs holds the right-hand side the solver was built from.
class DeviceSolver : public IterativeSolver {
protected:
    const MatrixCSR& a;
    DeviceBuffer<double> rhs;
    cas_solver* s = nullptr;

    static cas_solve_opts opts(cas_method method, int jacobi)
    {
        cas_solve_opts o;
        cas_solve_opts_default(&o);
        o.method = method;
        o.tol = 0;  // Iterate(n) runs exactly n steps
        o.max_iterations = 1 << 30;
        o.jacobi = jacobi;
        return o;
    }

public:
    DeviceSolver(const MatrixCSR& a, const Vector& rhs_host) : a(a), rhs(to_device_f64(rhs_host)) {}
    ~DeviceSolver() override { cas_solver_destroy(s); }
    DeviceSolver(const DeviceSolver&) = delete;
    DeviceSolver& operator=(const DeviceSolver&) = delete;

    void Iterate(int n = 1) override { check(cas_solver_iterate(s, n)); }
    float Residuum() const override
    {
        double r = 0;
        check(cas_solver_residuum(s, &r));
        return static_cast<float>(r);
    }
    Vector X() const override
    {
        DeviceBuffer<double> x(a.Cols());
        check(cas_solver_x(s, x.p));
        cudaDeviceSynchronize();
        return to_host_f32(x, a.Cols());
    }
    // Relative normal-equation residual ||A'(b - Ax)|| / ||A'b||, FP64.
    double RelativeResidual() const
    {
        double r = 0;
        check(cas_solver_rel_residual(s, &r));
        return r;
    }
};
}  // namespace detail

// PCG as FitWeights builds it (PatternFit/PatternFit.cpp:29-31):
//   DiagonalPreconditioner P(JacobiPreconditionerOfATA(A));
//   PCG solver(transposed(A) * A, P, x0, transposed(A) * b);
// The system matrix must be the lazy transposed(A) * A of a MatrixCSR; b' =
// A'b is the cols-length right-hand side, as in the reference.  P must be a
// DiagonalPreconditioner (Math/Solver.h:25-38), whatever its diagonal: its
// d is uploaded and applied on the device.  Any other Preconditioner throws
// std::invalid_argument (the device applies diagonal preconditioners only).
template <typename M>
class PCG;

template <>
class PCG<TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR>> final : public detail::DeviceSolver {
public:
    PCG(const TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR>& ata, const Preconditioner& P, Vector x0, Vector b)
        : DeviceSolver(ata.r, b)
    {
        if (ata.Rows() != ata.Cols()) throw std::runtime_error("Size mismatch.");
        if (ata.Cols() != x0.size()) throw std::runtime_error("Size mismatch.");
        if (ata.Rows() != b.size()) throw std::runtime_error("Size mismatch.");
        const auto* diag = dynamic_cast<const DiagonalPreconditioner*>(&P);
        if (!diag) throw std::invalid_argument("PCG: only a DiagonalPreconditioner is applied on the device");
        if (diag->d.size() != ata.Cols()) throw std::runtime_error("Size mismatch");
        cas_solve_opts o = opts(CAS_PCG, 1);
        auto dx0 = detail::to_device_f64(x0);
        auto dd = detail::to_device_f64(diag->d);
        check(cas_solver_create_normal_diag(a.device(), &o, rhs.p, dd.p, dx0.p, nullptr, &s));
    }
    // Error() = b' - A'A x (Math/Solver.h:115).
    Vector Error() const override
    {
        Vector r = (a * X()) * a;
        std::vector<double> hb(a.Cols());
        rhs.download(hb.data(), hb.size());
        for (size_t i = 0; i < r.size(); i++) r[i] = static_cast<float>(hb[i] - r[i]);
        return r;
    }
};

// CG on the same normal equations with P = I (Math/Solver.h:40-76).
template <typename M>
class CG;

template <>
class CG<TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR>> final : public detail::DeviceSolver {
public:
    CG(const TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR>& ata, Vector x0, Vector b) : DeviceSolver(ata.r, b)
    {
        if (ata.Cols() != ata.Rows() || ata.Cols() != x0.size() || ata.Rows() != b.size())
            throw std::runtime_error("Size mismatch.");
        cas_solve_opts o = opts(CAS_CG, 0);
        auto dx0 = detail::to_device_f64(x0);
        check(cas_solver_create_normal(a.device(), &o, rhs.p, dx0.p, nullptr, &s));
    }
    Vector Error() const override
    {
        Vector r = (a * X()) * a;
        std::vector<double> hb(a.Cols());
        rhs.download(hb.data(), hb.size());
        for (size_t i = 0; i < r.size(); i++) r[i] = static_cast<float>(hb[i] - r[i]);
        return r;
    }
};

// LSQR(A, x0, b) (Math/Solver.h:128-182) on the rows-length targets b.
template <typename M>
class LSQR;

template <>
class LSQR<MatrixCSR> final : public detail::DeviceSolver {
public:
    LSQR(const MatrixCSR& a, Vector x0, Vector b) : DeviceSolver(a, b)
    {
        if (a.Cols() != x0.size()) throw std::runtime_error("Size mismatch.");
        if (a.Rows() != b.size()) throw std::runtime_error("Size mismatch.");
        cas_solve_opts o = opts(CAS_LSQR, 0);
        auto dx0 = detail::to_device_f64(x0);
        check(cas_solver_create(a.device(), &o, rhs.p, dx0.p, nullptr, &s));
    }
    // Error() = b - A x (Math/Solver.h:180).
    Vector Error() const override
    {
        Vector r = a * X();
        std::vector<double> hb(a.Rows());
        rhs.download(hb.data(), hb.size());
        for (size_t i = 0; i < r.size(); i++) r[i] = static_cast<float>(hb[i] - r[i]);
        return r;
    }
};

// LSMR(A, x0, b) (Math/Solver.h:222-287) on the rows-length targets b.
// Residuum() is 0, as the reference's (:284).
template <typename M>
class LSMR;

template <>
class LSMR<MatrixCSR> final : public detail::DeviceSolver {
public:
    LSMR(const MatrixCSR& a, Vector x0, Vector b) : DeviceSolver(a, b)
    {
        if (a.Cols() != x0.size()) throw std::runtime_error("Size mismatch.");
        if (a.Rows() != b.size()) throw std::runtime_error("Size mismatch.");
        cas_solve_opts o = opts(CAS_LSMR, 0);
        auto dx0 = detail::to_device_f64(x0);
        check(cas_solver_create(a.device(), &o, rhs.p, dx0.p, nullptr, &s));
    }
    // Error() = b - A x (Math/Solver.h:286).
    Vector Error() const override
    {
        Vector r = a * X();
        std::vector<double> hb(a.Rows());
        rhs.download(hb.data(), hb.size());
        for (size_t i = 0; i < r.size(); i++) r[i] = static_cast<float>(hb[i] - r[i]);
        return r;
    }
};

// Class template argument deduction as in the reference's
// `PCG solver(transposed(A) * A, P, x0, b)`.
PCG(const TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR>&, const Preconditioner&, Vector, Vector)
    -> PCG<TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR>>;
CG(const TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR>&, Vector, Vector)
    -> CG<TwoMatrix<TransposedMatrix<MatrixCSR>, MatrixCSR>>;
LSQR(const MatrixCSR&, Vector, Vector) -> LSQR<MatrixCSR>;
LSMR(const MatrixCSR&, Vector, Vector) -> LSMR<MatrixCSR>;

// Pattern indexer (Pattern/Indexer.h:29-40).  Positions are {P, O} pairs.
class GroupIndexer {
    cas_patterns* p = nullptr;

public:
    int index_space_size = 0;

    explicit GroupIndexer(const std::vector<uint64_t>& pattern, cas_index_mode mode = CAS_INDEX_REFERENCE)
    {
        check(cas_patterns_create(pattern.data(), static_cast<int>(pattern.size()), mode, &p));
        index_space_size = static_cast<int>(cas_patterns_cols(p));
    }
    ~GroupIndexer() { cas_patterns_destroy(p); }
    GroupIndexer(const GroupIndexer&) = delete;
    GroupIndexer& operator=(const GroupIndexer&) = delete;

    const cas_patterns* handle() const noexcept { return p; }

    std::vector<uint64_t> Variations() const
    {
        std::vector<uint64_t> v(cas_patterns_nnz_per_row(p));
        check(cas_patterns_variations(p, v.data()));
        return v;
    }

    // Indices of many positions at once, row-major (positions: 2 words each).
    std::vector<uint32_t> Indices(std::span<const uint64_t> positions) const
    {
        const size_t n = positions.size() / 2, k = static_cast<size_t>(cas_patterns_nnz_per_row(p));
        detail::DeviceBuffer<uint64_t> dpos(positions.size());
        dpos.upload(positions.data(), positions.size());
        detail::DeviceBuffer<uint32_t> out(n * k);
        check(cas_index(p, dpos.p, static_cast<int64_t>(n), out.p, nullptr));
        std::vector<uint32_t> h(n * k);
        out.download(h.data(), h.size());
        return h;
    }

    // InsertIndices(Position, span) (Pattern/Indexer.cpp:413-422) for one position.
    void InsertIndices(uint64_t P, uint64_t O, std::span<uint32_t> location) const
    {
        const uint64_t pos[2] = {P, O};
        auto v = Indices(pos);
        if (location.size() < v.size()) throw std::runtime_error("Size mismatch.");
        std::memcpy(location.data(), v.data(), sizeof(uint32_t) * v.size());
    }
};

// FitWeights(pattern, positions, iterations) (PatternFit/PatternFit.cpp:7-39):
// positions are {P, O} pairs, scores one per position; `iterations`
// Jacobi-PCG steps from x0 = 0, as the reference.
inline Vector FitWeights(const std::vector<uint64_t>& pattern, std::span<const uint64_t> positions,
                         std::span<const float> scores, int iterations,
                         cas_index_mode mode = CAS_INDEX_REFERENCE)
{
    if (positions.size() != 2 * scores.size()) throw std::runtime_error("Size mismatch.");
    cas_patterns* p = nullptr;
    check(cas_patterns_create(pattern.data(), static_cast<int>(pattern.size()), mode, &p));
    const int64_t cols = cas_patterns_cols(p);
    cas_patterns_destroy(p);
    cas_solve_opts o;
    cas_solve_opts_default(&o);
    o.tol = 0;
    o.max_iterations = iterations;
    Vector w(static_cast<size_t>(cols));
    check(cas_fit_weights(pattern.data(), static_cast<int>(pattern.size()), mode, positions.data(), scores.data(),
                          static_cast<int64_t>(scores.size()), &o, w.data(), nullptr));
    return w;
}

// FitWeights to a tolerance instead of a fixed iteration count.
inline Vector FitWeightsToTolerance(const std::vector<uint64_t>& pattern, std::span<const uint64_t> positions,
                                    std::span<const float> scores, const cas_solve_opts& opts,
                                    cas_solve_report* report = nullptr, cas_index_mode mode = CAS_INDEX_REFERENCE)
{
    if (positions.size() != 2 * scores.size()) throw std::runtime_error("Size mismatch.");
    cas_patterns* p = nullptr;
    check(cas_patterns_create(pattern.data(), static_cast<int>(pattern.size()), mode, &p));
    const int64_t cols = cas_patterns_cols(p);
    cas_patterns_destroy(p);
    Vector w(static_cast<size_t>(cols));
    check(cas_fit_weights(pattern.data(), static_cast<int>(pattern.size()), mode, positions.data(), scores.data(),
                          static_cast<int64_t>(scores.size()), &opts, w.data(), report));
    return w;
}

}  // namespace cassandra_b200
