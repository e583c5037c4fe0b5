// jimwlk.hpp -- C++ adapter over libjimwlk that re-exposes the reference
// solver's classes and functions (config.h, field.h, matrix.h,
// mpi_fftw_class.h, MV_class.h, momenta.h, positions.h, mpi_class.h of
// ElsevierSoftwareX/SOFTX-D-21-00092) on device-resident fields, so that the
// body of main_optimized.cpp ports call for call.  Header-only; link with
// libjimwlk.so.
//
// What changes for a caller of the reference:
//  - fields live on one GPU and are constructed from a `device` (the context
//    that replaces mpi_class + momenta + positions + fftw2D set-up,
//    main_optimized.cpp:74-92) instead of (Nxl, Nyl); lfield and gfield are the
//    same type, since one GPU holds the whole lattice, and allgather is a copy;
//  - mpi_class, momenta and positions remain as empty types so that the
//    reference's signatures still compile;
//  - the Gaussian generators are counter based: the n-th call of
//    setMVModel draws MV slice n and the n-th call of generate_gaussian[...]
//    draws Langevin step n of the device's seed, the same sequential order as
//    the reference's generator, but reproducible;
//  - errors throw jimwlk::error (the reference returns 1 and goes on);
//  - prepare_A_and_B replaces the per-site loop of prepare_A_and_B_local
//    (main_optimized.cpp:287-300) by one call for all sites.
#pragma once

#include <complex>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/jimwlk.h"

namespace jimwlk {

struct error : std::runtime_error {
    jw_status status;
    error(jw_status s, const std::string& where)
        : std::runtime_error(where + ": " + jw_status_string(s)), status(s) {}
};

inline void check(jw_status s, const char* where) {
    if (s != JW_OK) throw error(s, where);
}

// config.h:38-42 (FIXED_COUPLING_CONSTANT is this library's fixed coupling,
// alpha_s folded into `step`).
enum Evolution { POSITION_EVOLUTION = JW_POSITION_EVOLUTION, MOMENTUM_EVOLUTION = JW_MOMENTUM_EVOLUTION };
enum Coupling {
    SQRT_COUPLING_CONSTANT = JW_SQRT_COUPLING_CONSTANT,
    NOISE_COUPLING_CONSTANT = JW_NOISE_COUPLING_CONSTANT,
    HATTA_COUPLING_CONSTANT = JW_HATTA_COUPLING_CONSTANT,
    FIXED_COUPLING_CONSTANT = JW_FIXED_COUPLING_CONSTANT
};
enum Kernel { LINEAR_KERNEL = JW_LINEAR_KERNEL, SIN_KERNEL = JW_SIN_KERNEL };

// class config (config.h:44-137); Nx = Ny is a run-time value.
class config {
public:
    int Nx, Ny, Nxl, Nyl;
    int stat;
    double mu, mass;
    int elementaryWilsonLines;
    std::string file_name;
    int langevin_steps, measurements;
    double step;
    Evolution EvolutionChoice;
    Coupling CouplingChoice;
    Kernel KernelChoice;
    uint64_t seed;

    explicit config(int N = 64) {
        jw_config c;
        check(jw_config_defaults(&c), "jw_config_defaults");
        c.Nx = c.Ny = N;
        from(c);
    }
    // config::read_config_from_file (config.h:76-136): the same grammar; the
    // lattice size is kept.
    int read_config_from_file(const std::string& path) {
        jw_config c = c_config();
        check(jw_config_read(&c, path.c_str()), "jw_config_read");
        from(c);
        return 1;
    }
    jw_config c_config() const {
        jw_config c;
        jw_config_defaults(&c);
        c.Nx = Nx;
        c.Ny = Ny;
        c.stat = stat;
        c.mu = mu;
        c.mass = mass;
        c.elementaryWilsonLines = elementaryWilsonLines;
        std::snprintf(c.file_name, sizeof c.file_name, "%s", file_name.c_str());
        c.langevin_steps = langevin_steps;
        c.measurements = measurements;
        c.step = step;
        c.EvolutionChoice = EvolutionChoice;
        c.CouplingChoice = CouplingChoice;
        c.KernelChoice = KernelChoice;
        c.seed = seed;
        return c;
    }

private:
    void from(const jw_config& c) {
        Nx = Nxl = c.Nx;
        Ny = Nyl = c.Ny;
        stat = c.stat;
        mu = c.mu;
        mass = c.mass;
        elementaryWilsonLines = c.elementaryWilsonLines;
        file_name = c.file_name;
        langevin_steps = c.langevin_steps;
        measurements = c.measurements;
        step = c.step;
        EvolutionChoice = static_cast<Evolution>(c.EvolutionChoice);
        CouplingChoice = static_cast<Coupling>(c.CouplingChoice);
        KernelChoice = static_cast<Kernel>(c.KernelChoice);
        seed = c.seed;
    }
};

// Single-GPU stand-ins for the reference's decomposition and tables.
class mpi_class {
public:
    mpi_class() = default;
    mpi_class(int, char**) {}
    int mpi_init(config*) { return 1; }
    int mpi_exchange_grid() { return 1; }
    int getPosX() const { return 0; }
    int getPosY() const { return 0; }
};
class momenta {
public:
    momenta(config*, mpi_class*) {}
    int set() { return 1; }
};
class positions {
public:
    positions(config*, mpi_class*) {}
    int set() { return 1; }
};

// MV_class (MV_class.h): the model's parameters.
class MV_class {
public:
    double g_parameter, mu_parameter;
    int Ny_parameter;
    MV_class(double g, double mu, int ny) : g_parameter(g), mu_parameter(mu), Ny_parameter(ny) {}
};

// One GPU context: device, stream, FFT tables and the noise counters.
class device {
public:
    explicit device(const config& cfg, int dev = 0) : N(cfg.Nx) {
        const jw_config c = cfg.c_config();
        check(jw_context_create(&c, dev, &ctx), "jw_context_create");
    }
    ~device() { jw_context_destroy(ctx); }
    device(const device&) = delete;
    device& operator=(const device&) = delete;
    // Waits for the device; throws on a flagged eigensolver failure or NaN.
    void sync() { check(jw_context_sync(ctx), "jw_context_sync"); }

    jw_context* ctx = nullptr;
    int N;
    uint64_t noise_step = 0;  // next Langevin step index
    int mv_slice = 0;         // next MV slice index
};

template <class T, int t>
class lfield {
    static_assert(std::is_same<T, double>::value, "device fields are FP64");
    static_assert(t == 1 || t == 9, "t is 1 or 9");

public:
    explicit lfield(device& d) : dev(&d) { check(jw_field_create(d.ctx, t, &f), "jw_field_create"); }
    lfield(const lfield& o) : dev(o.dev) {
        check(jw_field_create(dev->ctx, t, &f), "jw_field_create");
        check(jw_field_copy(f, o.f), "jw_field_copy");
    }
    lfield& operator=(const lfield& o) {  // field.h:301-318
        check(jw_field_copy(f, o.f), "jw_field_copy");
        return *this;
    }
    ~lfield() { jw_field_destroy(f); }

    int setToUnit() { check(jw_field_set_unit(f), "jw_field_set_unit"); return 1; }
    int setToZero() { check(jw_field_set_zero(f), "jw_field_set_zero"); return 1; }
    // field.h:683-757: the next MV slice of the device's stream.
    int setMVModel(MV_class* mv) {
        check(jw_set_mv_model(dev->ctx, f, dev->mv_slice++, mv->g_parameter, mv->mu_parameter, mv->Ny_parameter),
              "jw_set_mv_model");
        return 1;
    }
    int solvePoisson(double mass, double g, momenta* = nullptr) {  // field.h:867-877
        check(jw_solve_poisson(dev->ctx, f, mass, g), "jw_solve_poisson");
        return 1;
    }
    lfield& operator*=(const lfield& o) {  // field.h:337-365: V <- V exp(i f)
        check(jw_mul_exp(dev->ctx, f, o.f), "jw_mul_exp");
        return *this;
    }
    int trace(lfield<T, 1>* corr) {  // field.h:1375-1432
        check(jw_trace(dev->ctx, f, corr->f), "jw_trace");
        return 1;
    }
    int allgather(lfield* src, mpi_class* = nullptr) {
        *this = *src;
        return 1;
    }
    int average_and_symmetrize() {  // field.h:1460-1492
        check(jw_average_and_symmetrize(dev->ctx, f), "jw_average_and_symmetrize");
        return 1;
    }
    int reduce(lfield<T, 1>* sum, lfield<T, 1>* err, mpi_class* = nullptr) {  // field.h:1521-1536
        check(jw_reduce(dev->ctx, f, sum->f, err->f), "jw_reduce");
        return 1;
    }
    int reduce_hatta(lfield<T, 1>* sum, lfield<T, 1>* err, mpi_class*, int xr, int yr) {  // field.h:1538-1564
        check(jw_reduce_hatta(dev->ctx, f, sum->f, err->f, xr, yr), "jw_reduce_hatta");
        return 1;
    }
    int setCorrelationsForCouplingConstant(momenta* = nullptr) {  // field.h:1633-1651
        check(jw_set_correlations_for_coupling_constant(dev->ctx, f), "jw_set_correlations_for_coupling_constant");
        return 1;
    }
    template <class M>
    int multiplyByCholesky(M* mm) {  // field.h:1653-1689
        check(jw_multiply_by_cholesky(dev->ctx, f, mm->L), "jw_multiply_by_cholesky");
        return 1;
    }
    // Host copies in the reference layout u[(x*Ny + y)*t + k].
    std::vector<std::complex<T>> get() const {
        std::vector<std::complex<T>> u((size_t)dev->N * dev->N * t);
        check(jw_field_get(f, reinterpret_cast<double*>(u.data())), "jw_field_get");
        return u;
    }
    void set(const std::vector<std::complex<T>>& u) {
        if (u.size() != (size_t)dev->N * dev->N * t) throw error(JW_EINVAL, "lfield::set");
        check(jw_field_set(f, reinterpret_cast<const double*>(u.data())), "jw_field_set");
    }

    device* dev;
    jw_field* f = nullptr;
};

template <class T, int t>
using gfield = lfield<T, t>;

// gmatrix<T> holding the Cholesky factor (matrix.h:151-200).
template <class T>
class gmatrix {
public:
    explicit gmatrix(device& d) : dev(&d) {}
    ~gmatrix() { jw_cholesky_destroy(L); }
    gmatrix(const gmatrix&) = delete;
    gmatrix& operator=(const gmatrix&) = delete;
    int decompose(gfield<T, 1>* corr) {
        jw_cholesky_destroy(L);
        L = nullptr;
        check(jw_cholesky_decompose(dev->ctx, corr->f, &L), "jw_cholesky_decompose");
        return 1;
    }
    device* dev;
    jw_cholesky* L = nullptr;
};

// fftw2D (mpi_fftw_class.h:36-350).
class fftw2D {
public:
    explicit fftw2D(device& d) : dev(&d) {}
    int init2D() { return 1; }
    template <int t>
    int execute2D(lfield<double, t>* f, int dir) {
        check(jw_execute2D(dev->ctx, f->f, dir), "jw_execute2D");
        return 1;
    }
    device* dev;
};

// ---- field.h free functions
template <class T>
int generate_gaussian(lfield<T, 9>* xi_x, lfield<T, 9>* xi_y, mpi_class* = nullptr, config* = nullptr) {
    device* d = xi_x->dev;
    check(jw_generate_gaussian(d->ctx, xi_x->f, xi_y->f, d->noise_step++, 0), "jw_generate_gaussian");
    return 1;
}
template <class T>
int generate_gaussian_with_noise_coupling_constant(lfield<T, 9>* xi_x, lfield<T, 9>* xi_y, momenta* = nullptr,
                                                   mpi_class* = nullptr, config* = nullptr) {
    device* d = xi_x->dev;
    check(jw_generate_gaussian(d->ctx, xi_x->f, xi_y->f, d->noise_step++, 1), "jw_generate_gaussian");
    return 1;
}
template <class T>
int prepare_A_local(lfield<T, 9>* out, lfield<T, 9>* xi_x, lfield<T, 9>* xi_y, momenta*, mpi_class*, Coupling p,
                    Kernel k) {
    check(jw_prepare_A_local(out->dev->ctx, out->f, xi_x->f, xi_y->f, p, k), "jw_prepare_A_local");
    return 1;
}
template <class T>
int uxiulocal(lfield<T, 9>* ux, lfield<T, 9>* uy, lfield<T, 9>* uf, lfield<T, 9>* xi_x, lfield<T, 9>* xi_y) {
    check(jw_uxiulocal(ux->dev->ctx, ux->f, uy->f, uf->f, xi_x->f, xi_y->f), "jw_uxiulocal");
    return 1;
}
template <class T>
int update_uf(lfield<T, 9>* uf, lfield<T, 9>* B, lfield<T, 9>* A, double step) {
    check(jw_update_uf(uf->dev->ctx, uf->f, B->f, A->f, step), "jw_update_uf");
    return 1;
}
// prepare_A_and_B_local for every site (main_optimized.cpp:287-300).
template <class T>
int prepare_A_and_B(gfield<T, 9>* xi_x, gfield<T, 9>* xi_y, lfield<T, 9>* A, lfield<T, 9>* B, gfield<T, 9>* uf,
                    positions*, int rr, Coupling p, Kernel k) {
    check(jw_prepare_A_and_B(A->dev->ctx, A->f, B->f, xi_x->f, xi_y->f, uf->f, rr, p, k), "jw_prepare_A_and_B");
    return 1;
}
// print (field.h:2521-2547): appends to <file_name>_<Nx>_<Ny>_mpi1_r0.dat.
template <class T>
int print(int measurement, lfield<T, 1>* sum, lfield<T, 1>* err, momenta*, double x, mpi_class*,
          const std::string& file_name) {
    check(jw_print(sum->dev->ctx, measurement, sum->f, err->f, x, file_name.c_str()), "jw_print");
    return 1;
}

}  // namespace jimwlk
