// Tangent-linear (forward-mode) restatement of the oracle loop -- TEST
// INFRASTRUCTURE (oracle).  It differentiates the same FP64 loop as
// orc_step (monodomain.c: solve_monodomain's loop body,
// src/monodomain/monodomain_solver.c:616-925) for a TT2006 tissue with
// per-cell conductivity, along one direction in (conductivity, gKr scaling):
//
//   - the cell model: tt2006.c compiled a second time below with `double`
//     standing for a dual number (value, derivative), so the tangent runs the
//     very statements of orc_tt2006_step (ten_tusscher_2006_RS_CPU.c:100-351);
//   - the implicit solve A(sigma) v = alpha V*: the value by orc_pcg as in the
//     loop, the derivative by a second solve A dv = alpha dV* - dA v, where dA
//     comes from the derivative of the harmonic-mean face conductivity
//     2 s1 s2 / (s1 + s2) of every face (assembly_common.c:969-991), solved to
//     a relative residual of 1e-14.
//
// The result is the exact directional derivative of the loop's misfit (up to
// the solves' tolerances), against which the product's discrete adjoint is
// checked; the oracle's own central differences pin this file.
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "oracle.h"

namespace tl {

struct Dual {
    double v, d;
    Dual(double x = 0.0) : v(x), d(0.0) {}
    Dual(double x, double dx) : v(x), d(dx) {}
    Dual &operator+=(const Dual &o) { d += o.d; v += o.v; return *this; }
    Dual &operator-=(const Dual &o) { d -= o.d; v -= o.v; return *this; }
    Dual &operator*=(const Dual &o) { *this = Dual(v * o.v, d * o.v + v * o.d); return *this; }
    Dual &operator/=(const Dual &o) { *this = Dual(v / o.v, (d * o.v - v * o.d) / (o.v * o.v)); return *this; }
};

inline Dual operator+(const Dual &a, const Dual &b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(const Dual &a, const Dual &b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator*(const Dual &a, const Dual &b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(const Dual &a, const Dual &b) { return Dual(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
inline Dual operator-(const Dual &a) { return Dual(-a.v, -a.d); }
inline Dual operator+(const Dual &a) { return a; }
inline bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
inline bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
inline bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
inline bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
inline bool operator==(const Dual &a, const Dual &b) { return a.v == b.v; }
inline bool operator!=(const Dual &a, const Dual &b) { return a.v != b.v; }
inline Dual exp(const Dual &a) { const double e = ::exp(a.v); return Dual(e, e * a.d); }
inline Dual expm1(const Dual &a) { return Dual(::expm1(a.v), ::exp(a.v) * a.d); }
inline Dual log(const Dual &a) { return Dual(::log(a.v), a.d / a.v); }
inline Dual sqrt(const Dual &a) { const double r = ::sqrt(a.v); return Dual(r, a.d / (2.0 * r)); }
inline Dual fabs(const Dual &a) { return a.v < 0.0 ? -a : a; }
inline Dual pow(const Dual &a, const Dual &b) {
    const double p = ::pow(a.v, b.v);
    double dp = b.v * ::pow(a.v, b.v - 1.0) * a.d;
    if (b.d != 0.0) dp += p * ::log(a.v) * b.d;
    return Dual(p, dp);
}

// the cell model on dual numbers: the statements of tt2006.c (its includes
// are already in, so only its definitions are compiled here)
#define double Dual
#include "tt2006.c"
#undef double

}  // namespace tl

namespace {

double harmonic(double s1, double s2) {
    if (s1 != 0.0 && s2 != 0.0) return (2.0f * s1 * s2) / (s1 + s2);
    return 0.0;
}

// d harmonic(s1, s2) along (ds1, ds2)
double dharmonic(double s1, double s2, double ds1, double ds2) {
    if (s1 == 0.0 || s2 == 0.0) return 0.0;
    const double t = s1 + s2;
    return 2.0 * (s2 * s2 * ds1 + s1 * s1 * ds2) / (t * t);
}

}  // namespace

extern "C" int orc_tangent_misfit(const mb_monodomain_desc *d, int nsteps, int sample_every, int n_sensors,
                                  const int64_t *sensors, const double *target, const double *dsigma,
                                  const double *dgkr, double *loss, double *dloss) {
    using tl::Dual;
    if (!d || !loss || !dloss || nsteps < 0 || sample_every <= 0 || n_sensors < 0 || (n_sensors && (!sensors || !target)))
        return MB_ERR_ARG;
    if (d->model != MB_MODEL_TT2006) return MB_ERR_UNSUPPORTED;
    if (dsigma && (d->assembly != MB_ASSEMBLY_PER_CELL_SIGMA || !d->sigma_cell)) return MB_ERR_UNSUPPORTED;
    const int64_t ng = (int64_t)d->nx * d->ny * d->nz;
    std::vector<int32_t> cells((size_t)ng);
    orc_csr A;
    int rc = orc_assemble(d, &A, cells.data());
    if (rc) return rc;
    const int32_t n = A.n;
    std::vector<int32_t> row_of((size_t)ng, -1);
    for (int32_t c = 0; c < n; ++c) row_of[(size_t)cells[c]] = c;
    for (int i = 0; i < n_sensors; ++i)
        if (sensors[i] < 0 || sensors[i] >= ng || row_of[(size_t)sensors[i]] < 0) { orc_csr_free(&A); return MB_ERR_ARG; }

    // derivative of every face coefficient harmonic(s_c, s_j) * mult (the
    // off-diagonal entry is its negative, the diagonal holds their sum), so
    // (dA v)_c = sum over faces dcoef (v_c - v_j)
    std::vector<double> dcoef((size_t)A.row_ptr[n], 0.0);
    if (dsigma) {
        for (int32_t c = 0; c < n; ++c) {
            const double sc = d->sigma_cell[cells[c]], dsc = dsigma[cells[c]];
            for (int32_t k = A.row_ptr[c] + 1; k < A.row_ptr[c + 1]; ++k) {
                const int32_t j = A.col[k];
                const double sj = d->sigma_cell[cells[j]], dsj = dsigma[cells[j]];
                const double h = harmonic(sc, sj);
                if (h == 0.0) continue;
                const double mult = -A.val[k] / h;
                dcoef[(size_t)k] = dharmonic(sc, sj, dsc, dsj) * mult;
            }
        }
    }

    const int neq = ORC_TT_NEQ;
    const double alpha = (((d->beta * d->cm) / d->dt_pde) * (double)1.0e-8f) * (d->dx * d->dy * d->dz);
    int num_steps = (int)(d->dt_pde / d->dt_ode);
    if (num_steps < 1) num_steps = 1;
    const double dt = d->dt_ode;
    std::vector<Dual> sv((size_t)n * neq), scale;
    std::vector<double> v((size_t)n), dv((size_t)n, 0.0), b((size_t)n), rt((size_t)n), merged((size_t)n);
    std::vector<double> stim_val((size_t)MB_MAX_STIMS * n + 1, 0.0);
    double stim_start[MB_MAX_STIMS];
    if (d->current_scale || dgkr) {
        scale.assign((size_t)n * MB_NUM_SCALES, Dual(1.0));
        for (int32_t c = 0; c < n; ++c)
            for (int q = 0; q < MB_NUM_SCALES; ++q) {
                // the loop keeps the scalings as float
                const double s = d->current_scale ? (double)(float)d->current_scale[q * ng + cells[c]] : 1.0;
                scale[(size_t)c * MB_NUM_SCALES + q] = Dual(s, q == 1 && dgkr ? dgkr[cells[c]] : 0.0);
            }
    }
    const double v0 = !isnan(d->initial_v) ? d->initial_v : (double)-85.23f;
    for (int32_t c = 0; c < n; ++c) {
        Dual *y = &sv[(size_t)c * neq];
        if (d->initial_state)
            for (int q = 0; q < neq; ++q) y[q] = Dual(d->initial_state[q]);
        else tl::orc_tt2006_initial_state(y);
        v[c] = v0;
    }
    for (int k = 0; k < d->num_stims; ++k) stim_start[k] = d->stims[k].start;
    orc_stim_values(d, cells.data(), n, stim_val.data());

    double cur_time = 0.0, l = 0.0, dl = 0.0;
    const int nsamples = nsteps / sample_every;
    int sample = 0;
    for (int step = 0; step < nsteps; ++step) {
        if (cur_time > 0.0)
            for (int32_t c = 0; c < n; ++c) sv[(size_t)c * neq] = Dual(v[c], dv[c]);
        for (int32_t c = 0; c < n; ++c) merged[c] = 0.0;
        for (int k = 0; k < d->num_stims; ++k) {
            const double start = stim_start[k], dur = d->stims[k].duration, period = d->stims[k].period;
            double time = cur_time;
            for (int j = 0; j < num_steps; ++j) {
                if (time >= start && time <= start + dur)
                    for (int32_t c = 0; c < n; ++c) merged[c] += stim_val[(size_t)k * n + c];
                time += dt;
            }
            if (period > 0.0 && time >= start + period) stim_start[k] = start + period;
        }
        for (int32_t c = 0; c < n; ++c) {
            Dual *y = &sv[(size_t)c * neq];
            const Dual *sc = scale.empty() ? nullptr : &scale[(size_t)c * MB_NUM_SCALES];
            for (int j = 0; j < num_steps; ++j) tl::orc_tt2006_step(y, merged[c], dt, sc);
        }
        // b = alpha V*, the solve from x0 = V, then the tangent solve
        double rr = 0.0;
        for (int32_t c = 0; c < n; ++c) {
            const Dual bb = sv[(size_t)c * neq] * alpha;
            b[c] = bb.v;
            rt[c] = bb.d;
        }
        uint32_t its = 0;
        double err = 0.0;
        orc_pcg(&A, b.data(), v.data(), d->cg_tolerance, d->cg_max_iterations, d->use_preconditioner, &its, &err);
        if (isnan(err)) { orc_csr_free(&A); return MB_ERR_NAN; }
        for (int32_t c = 0; c < n; ++c) {
            double s = 0.0;
            for (int32_t k = A.row_ptr[c] + 1; k < A.row_ptr[c + 1]; ++k) s += dcoef[(size_t)k] * (v[c] - v[A.col[k]]);
            rt[c] -= s;
            rr += rt[c] * rt[c];
        }
        if (rr > 0.0) {
            orc_pcg(&A, rt.data(), dv.data(), 1e-28 * rr, 5000, 1, &its, &err);
            if (isnan(err)) { orc_csr_free(&A); return MB_ERR_NAN; }
        } else {
            for (int32_t c = 0; c < n; ++c) dv[c] = 0.0;
        }
        cur_time += d->dt_pde;
        if ((step + 1) % sample_every == 0 && sample < nsamples) {
            for (int i = 0; i < n_sensors; ++i) {
                const int32_t c = row_of[(size_t)sensors[i]];
                const double diff = v[c] - target[(size_t)sample * n_sensors + i];
                l += 0.5 * diff * diff;
                dl += diff * dv[c];
            }
            ++sample;
        }
    }
    orc_csr_free(&A);
    *loss = l;
    *dloss = dl;
    return MB_OK;
}
