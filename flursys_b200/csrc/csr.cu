// csr.cu — src/linear on the device: CsrMatrix::spmv_into, cg, pcg (Jacobi)
// and bicgstab (src/linear/{csr,solver,preconditioner,vector}.rs), FP64.
//
// The host validates the CSR arrays exactly as validate_csr (csr.rs:194-247)
// and the solve inputs as validate_solve_inputs (solver.rs:258-300), builds
// the Jacobi inverse diagonal with the errors of diagonal_entry /
// JacobiPreconditioner::new (csr.rs:67-82, preconditioner.rs:10-30), then
// runs one cooperative launch per solve. Device indices are 32-bit.
//
// CG/PCG keep the iteration order of solve_cg (solver.rs:62-153): the stop
// test ||r||_2 <= atol + rtol ||r0||_2 after each update, the breakdown tests
// |d.q| <= 1e-30, non-finite alpha, |rho| <= 1e-30 and non-finite beta. The
// direction update d = z + beta d is fused into the next SpMV: each gathered
// column forms z[col] + beta d_old[col] on the fly (bit-identical wherever it
// is formed) and the pass writes d_new for its own rows into a double buffer.
// BiCGSTAB follows bicgstab (solver.rs:155-256) with its early exit on ||s||.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.cuh"
#include "common.cuh"
#include "csr.cuh"

namespace flursys {

namespace {

constexpr int kBlock = 256;
constexpr int kParts = 4;

struct CsrDev {
    int n;
    const int *ro;
    const int *ci;
    const double *va;
    const double *inv_diag;  // PCG only
};

struct KrylovArgs {
    CsrDev a;
    const double *b;
    double *x;
    double *r, *z, *d0, *d1, *q;        // CG/PCG
    double *rh, *p, *v, *s, *t;         // BiCGSTAB
    double *partials;
    GridBarrier *bar;
    CsrResultDev *res;
    double atol, rtol;
    long long max_iters;
    int method;  // 0 cg, 1 pcg, 2 bicgstab
};

// Partial sums: every write -> grid barrier -> read group uses one of two
// column sets (kParts / 2 columns each) by the parity of `round`, so that a
// block never overwrites a set that a slower block may still be reading (the
// next write to the same set is one barrier further on). Each group's values
// are block-reduced through one set of block barriers (block_sum_n: the same
// shuffle tree per value as one reduction each).
template <int NV>
__device__ __forceinline__ void write_parts(double *part, int round, double (&v)[NV], double *red) {
    static_assert(NV <= kParts / 2, "one column set holds kParts / 2 values");
    block_sum_n<kBlock, NV>(v, red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) part[blockIdx.x * kParts + (round & 1) * (kParts / 2) + k] = v[k];
}
// Fixed-order sums over all blocks of the group's NV columns; ends the round.
template <int NV>
__device__ __forceinline__ void read_sums(const double *part, int &round, double (&out)[NV], double *red) {
    const int base = (round & 1) * (kParts / 2);
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock)
#pragma unroll
        for (int k = 0; k < NV; ++k) out[k] += __ldcg(part + b * kParts + base + k);
    block_sum_n<kBlock, NV>(out, red);
    ++round;
}

// Flags a non-finite SpMV row (first row wins through atomicMin).
__device__ __forceinline__ void flag_row(CsrResultDev *res, int row) {
    atomicMin(&res->bad_row, (unsigned long long)row);
}

__global__ void __launch_bounds__(kBlock) krylov_kernel(KrylovArgs k) {
    __shared__ double red[(kParts / 2) * (kBlock / 32)];
    int round = 0;  // partial-sum groups completed
    const int n = k.a.n;
    const int tid0 = blockIdx.x * kBlock + threadIdx.x, stride = gridDim.x * kBlock;
    const int *ro = k.a.ro, *ci = k.a.ci;
    const double *va = k.a.va;
    int error = 0, status = FLURSYS_LINEAR_MAX_ITERATIONS;
    long long iterations = 0;
    double initial = 0.0, fin = 0.0;
    auto spmv_row = [&](int row, auto val) -> double {
        double s = 0.0;
        for (int e = ro[row]; e < ro[row + 1]; ++e) s += va[e] * val(ci[e]);
        return s;
    };
    auto bail = [&]() -> bool { return k.res->bad_row != ~0ull; };

    // ---- r = b - A x (residual_into, vector.rs:115-138) ----
    {
        double srr = 0.0;
        for (int row = tid0; row < n; row += stride) {
            const double ax = spmv_row(row, [&](int c) { return k.x[c]; });
            if (!isfinite(ax)) flag_row(k.res, row);
            const double rv = k.b[row] - ax;
            k.r[row] = rv;
            if (k.method == 2) k.rh[row] = rv;
            srr += rv * rv;
        }
        double v[1] = {srr};
        write_parts<1>(k.partials, round, v, red);
    }
    if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
    double g0[1];
    read_sums<1>(k.partials, round, g0, red);
    if (bail()) { error = FLURSYS_ERR_NON_FINITE; goto done; }
    {
        const double rr0 = g0[0];
        initial = sqrt(rr0);
        fin = initial;
        if (!isfinite(initial)) { error = FLURSYS_ERR_NON_FINITE; goto done; }
    }
    {
        const double threshold = k.atol + k.rtol * initial;
        if (initial <= threshold) { status = FLURSYS_LINEAR_CONVERGED; goto done; }
        if (k.method != 2) {
            // ---- CG / PCG ----
            double srz = 0.0;
            for (int row = tid0; row < n; row += stride) {
                const double zv = k.method == 1 ? k.r[row] * k.a.inv_diag[row] : k.r[row];
                if (!isfinite(zv)) flag_row(k.res, row);
                k.z[row] = zv;
                srz += k.r[row] * zv;
            }
            {
                double v[1] = {srz};
                write_parts<1>(k.partials, round, v, red);
            }
            if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
            double g1[1];
            read_sums<1>(k.partials, round, g1, red);
            if (bail()) { error = FLURSYS_ERR_NON_FINITE; goto done; }
            double rho = g1[0];
            if (!isfinite(rho)) { error = FLURSYS_ERR_NON_FINITE; goto done; }
            double beta = 0.0;
            bool first = true;
            for (long long it = 1; it <= k.max_iters; ++it) {
                iterations = it;
                double *dcur = (it & 1) ? k.d0 : k.d1;
                const double *dold = (it & 1) ? k.d1 : k.d0;
                auto dval = [&](int c) { return first ? k.z[c] : k.z[c] + beta * dold[c]; };
                double sdq = 0.0;
                for (int row = tid0; row < n; row += stride) {
                    const double dr = dval(row);
                    const double qv = spmv_row(row, dval);
                    if (!isfinite(qv)) flag_row(k.res, row);
                    dcur[row] = dr;
                    k.q[row] = qv;
                    sdq += dr * qv;
                }
                {
                    double v[1] = {sdq};
                    write_parts<1>(k.partials, round, v, red);
                }
                if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
                double gd[1];
                read_sums<1>(k.partials, round, gd, red);
                if (bail()) { error = FLURSYS_ERR_NON_FINITE; break; }
                const double den = gd[0];
                if (!isfinite(den)) { error = FLURSYS_ERR_NON_FINITE; break; }  // dot() rejects it first
                if (fabs(den) <= 1.0e-30) { error = FLURSYS_ERR_BREAKDOWN; break; }
                const double alpha = rho / den;
                if (!isfinite(alpha)) { error = FLURSYS_ERR_BREAKDOWN; break; }
                double srr = 0.0, srz2 = 0.0;
                for (int row = tid0; row < n; row += stride) {
                    k.x[row] += alpha * dcur[row];
                    const double rv = k.r[row] - alpha * k.q[row];
                    k.r[row] = rv;
                    const double zv = k.method == 1 ? rv * k.a.inv_diag[row] : rv;
                    if (!isfinite(zv)) flag_row(k.res, row);
                    k.z[row] = zv;
                    srr += rv * rv;
                    srz2 += rv * zv;
                }
                {
                    double v[2] = {srr, srz2};
                    write_parts<2>(k.partials, round, v, red);
                }
                if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
                double gr[2];
                read_sums<2>(k.partials, round, gr, red);
                const double rn = sqrt(gr[0]);
                fin = rn;
                if (!isfinite(rn)) { error = FLURSYS_ERR_NON_FINITE; break; }
                if (rn <= threshold) { status = FLURSYS_LINEAR_CONVERGED; break; }
                if (bail()) { error = FLURSYS_ERR_NON_FINITE; break; }
                const double rho_new = gr[1];
                if (!isfinite(rho_new)) { error = FLURSYS_ERR_NON_FINITE; break; }
                if (fabs(rho) <= 1.0e-30) { error = FLURSYS_ERR_BREAKDOWN; break; }
                beta = rho_new / rho;
                if (!isfinite(beta)) { error = FLURSYS_ERR_BREAKDOWN; break; }
                rho = rho_new;
                first = false;
            }
            if (status != FLURSYS_LINEAR_CONVERGED) iterations = k.max_iters;
        } else {
            // ---- BiCGSTAB ----
            double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
            double rho = g0[0];  // r_hat = r0, so r_hat.r = ||r0||^2
            for (int row = tid0; row < n; row += stride) { k.p[row] = 0.0; k.v[row] = 0.0; }
            if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
            for (long long it = 1; it <= k.max_iters; ++it) {
                iterations = it;
                if (!isfinite(rho)) { error = FLURSYS_ERR_NON_FINITE; break; }
                if (fabs(rho) <= 1.0e-30) { error = FLURSYS_ERR_BREAKDOWN; break; }
                const double beta = (rho / rho_prev) * (alpha / omega);
                if (!isfinite(beta)) { error = FLURSYS_ERR_BREAKDOWN; break; }
                for (int row = tid0; row < n; row += stride) k.p[row] = k.r[row] + beta * (k.p[row] - omega * k.v[row]);
                if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
                double shv = 0.0;
                for (int row = tid0; row < n; row += stride) {
                    const double vv = spmv_row(row, [&](int c) { return k.p[c]; });
                    if (!isfinite(vv)) flag_row(k.res, row);
                    k.v[row] = vv;
                    shv += k.rh[row] * vv;
                }
                {
                    double v[1] = {shv};
                    write_parts<1>(k.partials, round, v, red);
                }
                if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
                double gv[1];
                read_sums<1>(k.partials, round, gv, red);
                if (bail()) { error = FLURSYS_ERR_NON_FINITE; break; }
                const double den = gv[0];
                if (!isfinite(den)) { error = FLURSYS_ERR_NON_FINITE; break; }
                if (fabs(den) <= 1.0e-30) { error = FLURSYS_ERR_BREAKDOWN; break; }
                alpha = rho / den;
                if (!isfinite(alpha)) { error = FLURSYS_ERR_BREAKDOWN; break; }
                double sss = 0.0;
                for (int row = tid0; row < n; row += stride) {
                    const double sv = k.r[row] - alpha * k.v[row];
                    k.s[row] = sv;
                    sss += sv * sv;
                }
                {
                    double v[1] = {sss};
                    write_parts<1>(k.partials, round, v, red);
                }
                if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
                double gs[1];
                read_sums<1>(k.partials, round, gs, red);
                const double sn = sqrt(gs[0]);
                if (!isfinite(sn)) { error = FLURSYS_ERR_NON_FINITE; break; }
                if (sn <= threshold) {
                    for (int row = tid0; row < n; row += stride) k.x[row] += alpha * k.p[row];
                    fin = sn;
                    status = FLURSYS_LINEAR_CONVERGED;
                    break;
                }
                double stt = 0.0, sts = 0.0;
                for (int row = tid0; row < n; row += stride) {
                    const double tv = spmv_row(row, [&](int c) { return k.s[c]; });
                    if (!isfinite(tv)) flag_row(k.res, row);
                    k.t[row] = tv;
                    stt += tv * tv;
                    sts += tv * k.s[row];
                }
                {
                    double v[2] = {stt, sts};
                    write_parts<2>(k.partials, round, v, red);
                }
                if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
                double gt[2];
                read_sums<2>(k.partials, round, gt, red);
                if (bail()) { error = FLURSYS_ERR_NON_FINITE; break; }
                const double tt = gt[0];
                const double ts_ = gt[1];
                if (!isfinite(tt) || !isfinite(ts_)) { error = FLURSYS_ERR_NON_FINITE; break; }
                if (fabs(tt) <= 1.0e-30) { error = FLURSYS_ERR_BREAKDOWN; break; }
                omega = ts_ / tt;
                if (!isfinite(omega) || fabs(omega) <= 1.0e-30) { error = FLURSYS_ERR_BREAKDOWN; break; }
                double srr = 0.0, shr = 0.0;
                for (int row = tid0; row < n; row += stride) {
                    k.x[row] += alpha * k.p[row] + omega * k.s[row];
                    const double rv = k.s[row] - omega * k.t[row];
                    k.r[row] = rv;
                    srr += rv * rv;
                    shr += k.rh[row] * rv;
                }
                {
                    double v[2] = {srr, shr};
                    write_parts<2>(k.partials, round, v, red);
                }
                if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
                double gq[2];
                read_sums<2>(k.partials, round, gq, red);
                const double rn = sqrt(gq[0]);
                fin = rn;
                if (!isfinite(rn)) { error = FLURSYS_ERR_NON_FINITE; break; }
                if (rn <= threshold) { status = FLURSYS_LINEAR_CONVERGED; break; }
                rho_prev = rho;
                rho = gq[1];
            }
            if (status != FLURSYS_LINEAR_CONVERGED) iterations = k.max_iters;
        }
    }
done:
    if (!grid_sync_report(k.bar, gridDim.x, &k.res->device_error)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        k.res->error = error;
        k.res->status = status;
        k.res->iterations = iterations;
        k.res->initial = initial;
        k.res->final_residual = fin;
        k.res->device_error = k.bar->error;
    }
}

__global__ void __launch_bounds__(kBlock) spmv_kernel(CsrDev a, const double *x, double *y, CsrResultDev *res) {
    for (int row = blockIdx.x * kBlock + threadIdx.x; row < a.n; row += gridDim.x * kBlock) {
        double s = 0.0;
        for (int e = a.ro[row]; e < a.ro[row + 1]; ++e) s += a.va[e] * x[a.ci[e]];
        if (!isfinite(s)) atomicMin(&res->bad_row, (unsigned long long)row);
        y[row] = s;
    }
}

// ---- host validation (csr.rs:194-247) ----
int32_t validate_csr_host(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t *ro, const int64_t *ci,
                          const double *va, std::string *msg) {
    if (!ro) { *msg = "row_offsets length must equal nrows + 1"; return FLURSYS_ERR_INVALID_CSR; }
    if (ro[0] != 0) { *msg = "first row offset must be zero"; return FLURSYS_ERR_INVALID_CSR; }
    if (ro[nrows] != nnz) { *msg = "last row offset must equal value count"; return FLURSYS_ERR_INVALID_CSR; }
    for (int64_t r = 0; r < nrows; ++r) {
        if (ro[r] > ro[r + 1]) { *msg = "row offsets must be monotonic"; return FLURSYS_ERR_INVALID_CSR; }
        for (int64_t e = ro[r] + 1; e < ro[r + 1]; ++e)
            if (ci[e - 1] >= ci[e]) { *msg = "row columns must be strictly ascending"; return FLURSYS_ERR_INVALID_CSR; }
    }
    for (int64_t e = 0; e < nnz; ++e)
        if (ci[e] < 0 || ci[e] >= ncols) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "column %lld at entry %lld exceeds ncols", (long long)ci[e], (long long)e);
            *msg = buf;
            return FLURSYS_ERR_INVALID_CSR;
        }
    for (int64_t e = 0; e < nnz; ++e)
        if (!std::isfinite(va[e])) {
            char buf[96];
            std::snprintf(buf, sizeof buf, "non-finite matrix value at index %lld", (long long)e);
            *msg = buf;
            return FLURSYS_ERR_NON_FINITE;
        }
    return FLURSYS_OK;
}

struct DeviceCsr {
    int *ro = nullptr, *ci = nullptr;
    double *va = nullptr;
    cudaError_t upload(int64_t nrows, int64_t nnz, const int64_t *ro64, const int64_t *ci64, const double *va64,
                       cudaStream_t st) {
        std::vector<int> h_ro(nrows + 1), h_ci(std::max<int64_t>(nnz, 1));
        for (int64_t r = 0; r <= nrows; ++r) h_ro[r] = (int)ro64[r];
        for (int64_t e = 0; e < nnz; ++e) h_ci[e] = (int)ci64[e];
        cudaError_t e = cudaMalloc(&ro, sizeof(int) * (nrows + 1));
        if (e == cudaSuccess) e = cudaMalloc(&ci, sizeof(int) * std::max<int64_t>(nnz, 1));
        if (e == cudaSuccess) e = cudaMalloc(&va, sizeof(double) * std::max<int64_t>(nnz, 1));
        if (e == cudaSuccess) e = cudaMemcpyAsync(ro, h_ro.data(), sizeof(int) * (nrows + 1), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(ci, h_ci.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(va, va64, sizeof(double) * nnz, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host staging vectors die at return
        return e;
    }
    ~DeviceCsr() {
        cudaFree(ro);
        cudaFree(ci);
        cudaFree(va);
    }
};

int32_t csr_solve(int method, int64_t n, int64_t nnz, const int64_t *ro, const int64_t *ci, const double *va,
                  const double *rhs, double *x, const FlursysLinearSolverOptions *opt, FlursysLinearSolveReport *rep) {
    std::string msg;
    if (n < 0 || nnz < 0 || !ro || (nnz > 0 && (!ci || !va)) || (n > 0 && (!rhs || !x)) || !opt) {
        set_global_error("null argument or negative size");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    if (n >= (1LL << 31) || nnz >= (1LL << 31)) {
        set_global_error("matrix too large for 32-bit device indices");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    int32_t st = validate_csr_host(n, n, nnz, ro, ci, va, &msg);
    if (st) { set_global_error("invalid CSR matrix: " + msg); return st; }
    // validate_solve_inputs (solver.rs:258-300)
    if (!std::isfinite(opt->absolute_tolerance) || opt->absolute_tolerance < 0.0 ||
        !std::isfinite(opt->relative_tolerance) || opt->relative_tolerance < 0.0) {
        set_global_error("iterative solver breakdown: invalid solver tolerance");
        return FLURSYS_ERR_BREAKDOWN;
    }
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(rhs[i])) { set_global_error("non-finite solver vector value"); return FLURSYS_ERR_NON_FINITE; }
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(x[i])) { set_global_error("non-finite solver vector value"); return FLURSYS_ERR_NON_FINITE; }
    std::vector<double> inv;
    if (method == 1) {
        inv.resize(n);
        for (int64_t r = 0; r < n; ++r) {
            const int64_t *b = ci + ro[r], *e = ci + ro[r + 1];
            const int64_t *f = std::lower_bound(b, e, r);
            char buf[96];
            if (f == e || *f != r) {
                std::snprintf(buf, sizeof buf, "missing diagonal entry in row %lld", (long long)r);
                set_global_error(buf);
                return FLURSYS_ERR_MISSING_DIAGONAL;
            }
            const double d = va[ro[r] + (f - b)];
            if (d == 0.0) {
                std::snprintf(buf, sizeof buf, "zero diagonal entry in row %lld", (long long)r);
                set_global_error(buf);
                return FLURSYS_ERR_ZERO_DIAGONAL;
            }
            inv[r] = 1.0 / d;
            if (!std::isfinite(inv[r])) { set_global_error("non-finite inverse diagonal"); return FLURSYS_ERR_NON_FINITE; }
        }
    }
    if (n == 0) {
        if (rep) *rep = FlursysLinearSolveReport{FLURSYS_LINEAR_CONVERGED, 0, 0, 0.0, 0.0, 0.0};
        return FLURSYS_OK;
    }
    int device = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, krylov_kernel, kBlock, 0);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * per_sm, (n + kBlock * 4 - 1) / (kBlock * 4)));
    cudaStream_t stream;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return FLURSYS_ERR_CUDA;
    DeviceCsr A;
    std::vector<double *> bufs;
    auto alloc = [&](double **p, size_t cnt, cudaError_t *e) {
        if (*e == cudaSuccess) *e = cudaMalloc(p, sizeof(double) * std::max<size_t>(cnt, 1));
        if (*e == cudaSuccess) bufs.push_back(*p);
    };
    KrylovArgs k{};
    cudaError_t e = A.upload(n, nnz, ro, ci, va, stream);
    double *dinv = nullptr, *db = nullptr, *dx = nullptr;
    alloc(&db, n, &e); alloc(&dx, n, &e);
    alloc(&k.r, n, &e); alloc(&k.z, n, &e); alloc(&k.d0, n, &e); alloc(&k.d1, n, &e); alloc(&k.q, n, &e);
    if (method == 2) { alloc(&k.rh, n, &e); alloc(&k.p, n, &e); alloc(&k.v, n, &e); alloc(&k.s, n, &e); alloc(&k.t, n, &e); }
    if (method == 1) alloc(&dinv, n, &e);
    alloc(&k.partials, (size_t)grid * kParts, &e);
    GridBarrier *bar = nullptr;
    CsrResultDev *dres = nullptr, *hres = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&bar, sizeof(GridBarrier));
    if (e == cudaSuccess) e = cudaMalloc(&dres, sizeof(CsrResultDev));
    if (e == cudaSuccess) e = cudaMallocHost(&hres, sizeof(CsrResultDev));
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && method == 1) e = cudaMemcpyAsync(dinv, inv.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(bar, 0, sizeof(GridBarrier), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dres, 0xff, sizeof(CsrResultDev), stream);
    int32_t status = FLURSYS_OK;
    if (e == cudaSuccess) {
        k.a = CsrDev{(int)n, A.ro, A.ci, A.va, dinv};
        k.b = db;
        k.x = dx;
        k.bar = bar;
        k.res = dres;
        k.atol = opt->absolute_tolerance;
        k.rtol = opt->relative_tolerance;
        k.max_iters = opt->max_iterations;
        k.method = method;
        void *params[] = {&k};
        e = cudaLaunchCooperativeKernel((const void *)krylov_kernel, dim3(grid), dim3(kBlock), params, 0, stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hres, dres, sizeof(CsrResultDev), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    std::string err;
    if (e != cudaSuccess) {
        status = set_cuda_error(&err, e, "CSR solve");
    } else if (hres->device_error & kDevErrBarrierTimeout) {
        status = FLURSYS_ERR_TIMEOUT;
        err = "CSR solve: a device grid barrier timed out";
    } else if (hres->error == FLURSYS_ERR_NON_FINITE) {
        status = FLURSYS_ERR_NON_FINITE;
        char buf[96];
        std::snprintf(buf, sizeof buf, "non-finite SpMV output value at index %llu", (unsigned long long)hres->bad_row);
        err = hres->bad_row != ~0ull ? buf : "non-finite solver value";
    } else if (hres->error == FLURSYS_ERR_BREAKDOWN) {
        status = FLURSYS_ERR_BREAKDOWN;
        err = "iterative solver breakdown";
    } else if (rep) {
        rep->status = hres->status;
        rep->reserved = 0;
        rep->iterations = hres->iterations;
        rep->initial_residual = hres->initial;
        rep->final_residual = hres->final_residual;
        rep->relative_residual = hres->initial == 0.0 ? 0.0 : hres->final_residual / hres->initial;
    }
    for (double *p : bufs) cudaFree(p);
    cudaFree(bar);
    cudaFree(dres);
    if (hres) cudaFreeHost(hres);
    cudaStreamDestroy(stream);
    if (status) set_global_error(err);
    return status;
}

// 1/diag of each row (ascending columns); error bit on a missing or zero diagonal.
__global__ void jacobi_inverse_kernel(int n, const int *ro, const int *ci, const double *va, double *inv,
                                      CsrResultDev *res) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        double d = 0.0;
        bool found = false;
        for (int e = ro[r]; e < ro[r + 1]; ++e)
            if (ci[e] == r) { d = va[e]; found = true; break; }
        if (!found || d == 0.0) {
            atomicCAS(&res->error, 0, found ? FLURSYS_ERR_ZERO_DIAGONAL : FLURSYS_ERR_MISSING_DIAGONAL);
            inv[r] = 0.0;
        } else {
            inv[r] = 1.0 / d;
        }
    }
}

}  // namespace

cudaError_t CsrDeviceWork::ensure(int n_, int device) {
    if (vec && n_ <= n) return cudaSuccess;
    release();
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, krylov_kernel, kBlock, 0);
    if (e != cudaSuccess) return e;
    grid = (int)std::max<long long>(1, std::min<long long>((long long)sms * per_sm, ((long long)n_ + kBlock * 4 - 1) / (kBlock * 4)));
    e = cudaMalloc(&vec, sizeof(double) * 10 * (size_t)std::max(n_, 1));
    if (e == cudaSuccess) e = cudaMalloc(&partials, sizeof(double) * kParts * (size_t)grid);
    if (e == cudaSuccess) e = cudaMalloc(&inv_diag, sizeof(double) * (size_t)std::max(n_, 1));
    if (e == cudaSuccess) e = cudaMalloc(&bar, sizeof(GridBarrier));
    if (e == cudaSuccess) e = cudaMalloc(&res, 2 * sizeof(CsrResultDev));   // [0] solve, [1] Jacobi set-up
    if (e == cudaSuccess) e = cudaMallocHost(&hres, 2 * sizeof(CsrResultDev));
    if (e == cudaSuccess) n = n_;
    return e;
}

void CsrDeviceWork::release() {
    cudaFree(vec); cudaFree(partials); cudaFree(inv_diag); cudaFree(bar); cudaFree(res);
    if (hres) cudaFreeHost(hres);
    vec = partials = inv_diag = nullptr;
    bar = nullptr;
    res = hres = nullptr;
    n = grid = 0;
}

cudaError_t csr_device_launch(int method, int n, const int *ro, const int *ci, const double *va, const double *b,
                              double *x, double atol, double rtol, long long max_iters, CsrDeviceWork &w,
                              cudaStream_t st) {
    KrylovArgs k{};
    double *v = w.vec;
    k.r = v; k.z = v + (size_t)n; k.d0 = v + 2 * (size_t)n; k.d1 = v + 3 * (size_t)n; k.q = v + 4 * (size_t)n;
    k.rh = v + 5 * (size_t)n; k.p = v + 6 * (size_t)n; k.v = v + 7 * (size_t)n; k.s = v + 8 * (size_t)n;
    k.t = v + 9 * (size_t)n;
    k.partials = w.partials;
    k.bar = w.bar;
    k.res = w.res;
    k.atol = atol;
    k.rtol = rtol;
    k.max_iters = max_iters;
    k.method = method;
    k.a = CsrDev{n, ro, ci, va, method == 1 ? w.inv_diag : nullptr};
    k.b = b;
    k.x = x;
    cudaError_t e = cudaMemsetAsync(w.bar, 0, sizeof(GridBarrier), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.res, 0xff, sizeof(CsrResultDev), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.res + 1, 0, sizeof(CsrResultDev), st);
    if (e == cudaSuccess && method == 1) {
        jacobi_inverse_kernel<<<std::min(1024, (n + 255) / 256), 256, 0, st>>>(n, ro, ci, va, w.inv_diag, w.res + 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        void *params[] = {&k};
        e = cudaLaunchCooperativeKernel((const void *)krylov_kernel, dim3(w.grid), dim3(kBlock), params, 0, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(w.hres, w.res, 2 * sizeof(CsrResultDev), cudaMemcpyDeviceToHost, st);
    return e;
}

int32_t csr_device_status(const CsrResultDev *rr, FlursysLinearSolveReport *rep, std::string *err) {
    const CsrResultDev &r = rr[0];
    if (rr[1].error == FLURSYS_ERR_MISSING_DIAGONAL || rr[1].error == FLURSYS_ERR_ZERO_DIAGONAL) {
        *err = rr[1].error == FLURSYS_ERR_ZERO_DIAGONAL ? "zero diagonal entry" : "missing diagonal entry";
        return rr[1].error;
    }
    if (r.device_error & kDevErrBarrierTimeout) {
        *err = "CSR solve: a device grid barrier timed out";
        return FLURSYS_ERR_TIMEOUT;
    }
    if (r.error == FLURSYS_ERR_NON_FINITE) {
        *err = "non-finite solver value";
        return FLURSYS_ERR_NON_FINITE;
    }
    if (r.error == FLURSYS_ERR_BREAKDOWN) {
        *err = "iterative solver breakdown";
        return FLURSYS_ERR_BREAKDOWN;
    }
    if (rep) {
        rep->status = r.status;
        rep->reserved = 0;
        rep->iterations = r.iterations;
        rep->initial_residual = r.initial;
        rep->final_residual = r.final_residual;
        rep->relative_residual = r.initial == 0.0 ? 0.0 : r.final_residual / r.initial;
    }
    return FLURSYS_OK;
}

}  // namespace flursys

using namespace flursys;

extern "C" {

int32_t flursys_cuda_csr_cg(int64_t n, int64_t nnz, const int64_t *ro, const int64_t *ci, const double *va,
                            const double *rhs, double *x, const FlursysLinearSolverOptions *o,
                            FlursysLinearSolveReport *rep) {
    return csr_solve(0, n, nnz, ro, ci, va, rhs, x, o, rep);
}
int32_t flursys_cuda_csr_pcg(int64_t n, int64_t nnz, const int64_t *ro, const int64_t *ci, const double *va,
                             const double *rhs, double *x, const FlursysLinearSolverOptions *o,
                             FlursysLinearSolveReport *rep) {
    return csr_solve(1, n, nnz, ro, ci, va, rhs, x, o, rep);
}
int32_t flursys_cuda_csr_bicgstab(int64_t n, int64_t nnz, const int64_t *ro, const int64_t *ci, const double *va,
                                  const double *rhs, double *x, const FlursysLinearSolverOptions *o,
                                  FlursysLinearSolveReport *rep) {
    return csr_solve(2, n, nnz, ro, ci, va, rhs, x, o, rep);
}

int32_t flursys_cuda_csr_spmv(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t *ro, const int64_t *ci,
                              const double *va, const double *input, double *output) {
    std::string msg;
    if (nrows < 0 || ncols < 0 || nnz < 0 || !ro || (nnz > 0 && (!ci || !va)) || (ncols > 0 && !input) ||
        (nrows > 0 && !output)) {
        set_global_error("null argument or negative size");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    if (nrows >= (1LL << 31) || ncols >= (1LL << 31) || nnz >= (1LL << 31)) {
        set_global_error("matrix too large for 32-bit device indices");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    int32_t st = validate_csr_host(nrows, ncols, nnz, ro, ci, va, &msg);
    if (st) { set_global_error("invalid CSR matrix: " + msg); return st; }
    if (nrows == 0) return FLURSYS_OK;
    cudaStream_t stream;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return FLURSYS_ERR_CUDA;
    DeviceCsr A;
    double *dxv = nullptr, *dy = nullptr;
    CsrResultDev *dres = nullptr, hres{};
    cudaError_t e = A.upload(nrows, nnz, ro, ci, va, stream);
    if (e == cudaSuccess) e = cudaMalloc(&dxv, sizeof(double) * std::max<int64_t>(ncols, 1));
    if (e == cudaSuccess) e = cudaMalloc(&dy, sizeof(double) * nrows);
    if (e == cudaSuccess) e = cudaMalloc(&dres, sizeof(CsrResultDev));
    if (e == cudaSuccess) e = cudaMemsetAsync(dres, 0xff, sizeof(CsrResultDev), stream);
    if (e == cudaSuccess && ncols) e = cudaMemcpyAsync(dxv, input, sizeof(double) * ncols, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        int sms = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * 8, (nrows + kBlock - 1) / kBlock));
        spmv_kernel<<<grid, kBlock, 0, stream>>>(CsrDev{(int)nrows, A.ro, A.ci, A.va, nullptr}, dxv, dy, dres);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hres, dres, sizeof(CsrResultDev), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(output, dy, sizeof(double) * nrows, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    int32_t status = FLURSYS_OK;
    std::string err;
    if (e != cudaSuccess) {
        status = set_cuda_error(&err, e, "CSR SpMV");
    } else if (hres.bad_row != ~0ull) {
        char buf[96];
        std::snprintf(buf, sizeof buf, "non-finite SpMV output value at index %llu", (unsigned long long)hres.bad_row);
        err = buf;
        status = FLURSYS_ERR_NON_FINITE;
    }
    cudaFree(dxv);
    cudaFree(dy);
    cudaFree(dres);
    cudaStreamDestroy(stream);
    if (status) set_global_error(err);
    return status;
}

}  // extern "C"
