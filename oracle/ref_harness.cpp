/*
 * Reference harness (oracle test infrastructure only): the reference solver's
 * OWN code -- field.h, su3_matrix.h, zheevh3-C-1.1/*.cpp, mpi_fftw_class.h,
 * momenta.h, positions.h, matrix.h, config.h, mpi_init.cpp,
 * mpi_exchange_grid.cpp -- compiled unmodified from the reference tree, with
 *   - shim/mpi.h, shim/fftw3.h, shim/fftw3-mpi.h (single rank, project FFT),
 *   - shim/jw_inject.h (deterministic injected Gaussians),
 *   - the compile-time lattice size Nx = Ny = JW_N (config.h:31-32 fixes 64;
 *     this file redefines the macros after config.h's include guard is set),
 * and exposed through extern "C" entry points so that tests can call the
 * reference's functions on identical inputs.  Built per lattice size into
 * oracle/_ref/libref_<N>.so by oracle/Makefile.  Nothing here is part of the
 * product library.
 *
 * Field arrays cross this boundary in the reference's own layout: site-major
 * interleaved complex, element k of site (x, y) at [(x*N + y)*t + k]
 * (field.h:73, 170-173), i.e. 2*t*N*N doubles per field.
 */
#include <complex>
#include <string.h>

#include "jw_inject.h"

#include "jw_ref_config.h"

#include "su3_matrix.h"
#include "matrix.h"
#include "field.h"
#include "mpi_fftw_class.h"
#include "momenta.h"
#include "positions.h"
#include "MV_class.h"
#include "mpi_init.cpp"
#include "mpi_exchange_grid.cpp"

namespace {

struct RefContext {
    config* cnfg = nullptr;
    mpi_class* mpi = nullptr;
    momenta* mom = nullptr;
    positions* pos = nullptr;
    fftw2D* fft = nullptr;
};

RefContext& ctx() {
    static RefContext c;
    return c;
}

/* main_optimized.cpp:68-92 with a 1x1 process grid. */
void ensure_init(const char* config_path) {
    RefContext& c = ctx();
    if (c.cnfg) return;
    c.cnfg = new config;
    if (config_path && config_path[0]) c.cnfg->read_config_from_file(config_path);
    static char a0[] = "ref", a1[] = "1", a2[] = "1";
    static char* argv[] = {a0, a1, a2, nullptr};
    c.mpi = new mpi_class(3, argv);
    c.mpi->mpi_init(c.cnfg);
    c.mpi->mpi_exchange_grid();
    c.mom = new momenta(c.cnfg, c.mpi);
    c.mom->set();
    c.pos = new positions(c.cnfg, c.mpi);
    c.pos->set();
    c.fft = new fftw2D(c.cnfg);
    c.fft->init2D();
}

template <int t>
void load(lfield<double, t>& f, const double* src) {
    memcpy((void*)f.u, src, sizeof(double) * 2 * t * Nx * Ny);
}
template <int t>
void store(const lfield<double, t>& f, double* dst) {
    memcpy(dst, (const void*)f.u, sizeof(double) * 2 * t * Nx * Ny);
}

}  // namespace

extern "C" {

int ref_N(void) { return Nx; }

/* Reads a config file in the reference grammar (config.h:76-136); "" keeps
 * the class defaults (config.h:60-73).  Must come before any other call. */
int ref_init(const char* config_path) {
    if (ctx().cnfg) return -1;
    ensure_init(config_path);
    return 0;
}

/* Parsed values, as the reference holds them after read_config_from_file. */
void ref_config(double* out_d, int* out_i) {
    ensure_init(nullptr);
    config* c = ctx().cnfg;
    out_d[0] = c->mu;
    out_d[1] = c->mass;
    out_d[2] = c->step;
    out_i[0] = c->stat;
    out_i[1] = c->elementaryWilsonLines;
    out_i[2] = c->langevin_steps;
    out_i[3] = c->measurements;
    out_i[4] = (int)c->EvolutionChoice;
    out_i[5] = (int)c->CouplingChoice;
    out_i[6] = (int)c->KernelChoice;
}

void ref_set_injection(const double* z, long n) { jw_inject_set(z, n); }
long ref_injection_consumed(void) { return jw_inject_global().pos; }

/* fftw2D::execute2D (mpi_fftw_class.h:191-315); t = 1 or 9, dir 1 = X->K. */
void ref_execute2D(double* data, int t, int dir) {
    ensure_init(nullptr);
    if (t == 9) {
        lfield<double, 9> f(Nx, Ny);
        load(f, data);
        ctx().fft->execute2D(&f, dir);
        store(f, data);
    } else {
        lfield<double, 1> f(Nx, Ny);
        load(f, data);
        ctx().fft->execute2D(&f, dir);
        store(f, data);
    }
}

/* generate_gaussian (field.h:2116-2243) or, with_coupling != 0,
 * generate_gaussian_with_noise_coupling_constant (field.h:2245-2365);
 * Gaussians come from the injected stream, 16 per site. */
void ref_generate_gaussian(double* xi_x, double* xi_y, int with_coupling) {
    ensure_init(nullptr);
    lfield<double, 9> fx(Nx, Ny), fy(Nx, Ny);
    if (with_coupling)
        generate_gaussian_with_noise_coupling_constant(&fx, &fy, ctx().mom, ctx().mpi, ctx().cnfg);
    else
        generate_gaussian(&fx, &fy, ctx().mpi, ctx().cnfg);
    store(fx, xi_x);
    store(fy, xi_y);
}

/* lfield::setMVModel (field.h:683-757) with the injected stream, 8 per site. */
void ref_set_mv_model(double* f_out, double g, double mu, int ny_slices) {
    ensure_init(nullptr);
    MV_class mv(g, mu, ny_slices);
    lfield<double, 9> f(Nx, Ny);
    f.setMVModel(&mv);
    store(f, f_out);
}

/* lfield::solvePoisson (field.h:867-877). */
void ref_solve_poisson(double* f_io, double mass, double g) {
    ensure_init(nullptr);
    lfield<double, 9> f(Nx, Ny);
    load(f, f_io);
    f.solvePoisson(mass, g, ctx().mom);
    store(f, f_io);
}

/* lfield::operator*= (field.h:337-365): V <- V * exp(+i f). */
void ref_mul_exp(double* V_io, const double* f_in) {
    ensure_init(nullptr);
    lfield<double, 9> V(Nx, Ny), f(Nx, Ny);
    load(V, V_io);
    load(f, f_in);
    V *= f;
    store(V, V_io);
}

/* prepare_A_local (field.h:1998-2075). */
void ref_prepare_A_local(double* A_out, const double* xi_x, const double* xi_y, int coupling, int kernel) {
    ensure_init(nullptr);
    lfield<double, 9> A(Nx, Ny), fx(Nx, Ny), fy(Nx, Ny);
    load(fx, xi_x);
    load(fy, xi_y);
    prepare_A_local(&A, &fx, &fy, ctx().mom, ctx().mpi, (Coupling)coupling, (Kernel)kernel);
    store(A, A_out);
}

/* uxiulocal (field.h:1892-1933). */
void ref_uxiulocal(double* ux, double* uy, const double* V, const double* xi_x, const double* xi_y) {
    ensure_init(nullptr);
    lfield<double, 9> a(Nx, Ny), b(Nx, Ny), u(Nx, Ny), fx(Nx, Ny), fy(Nx, Ny);
    load(u, V);
    load(fx, xi_x);
    load(fy, xi_y);
    uxiulocal(&a, &b, &u, &fx, &fy);
    store(a, ux);
    store(b, uy);
}

/* update_uf (field.h:1966-1996). */
void ref_update_uf(double* V_io, const double* B, const double* A, double step) {
    ensure_init(nullptr);
    lfield<double, 9> u(Nx, Ny), b(Nx, Ny), a(Nx, Ny);
    load(u, V_io);
    load(b, B);
    load(a, A);
    update_uf(&u, &b, &a, step);
    store(u, V_io);
}

/* su3_matrix::exponentiate (su3_matrix.h:173-253) on n matrices of 9 complex;
 * returns the number of eigensolver failures (function_zheevh3 status != 0). */
int ref_su3_exponentiate(double* m, long n, double sign) {
    int bad = 0;
    for (long s = 0; s < n; ++s) {
        su3_matrix<double> A;
        for (int k = 0; k < 9; ++k) A.m[k] = std::complex<double>(m[18 * s + 2 * k], m[18 * s + 2 * k + 1]);
        if (A.exponentiate(sign) != 0) ++bad;
        for (int k = 0; k < 9; ++k) {
            m[18 * s + 2 * k] = A.m[k].real();
            m[18 * s + 2 * k + 1] = A.m[k].imag();
        }
    }
    return bad;
}

/* The MV initial condition of main_optimized.cpp:88, 178-191:
 * MV_class(1, mu/Nx, elementaryWilsonLines); uf = 1; per slice setMVModel,
 * execute2D(+), solvePoisson(mass*g^2*mu_MV, g), execute2D(-), uf *= f. */
void ref_initial_condition(double* V_out) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    MV_class MVmodel(1.0, cnfg->mu / Nx, cnfg->elementaryWilsonLines);
    lfield<double, 9> f(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 9> uf(cnfg->Nxl, cnfg->Nyl);
    uf.setToUnit();
    for (int i = 0; i < MVmodel.Ny_parameter; i++) {
        f.setMVModel(&MVmodel);
        ctx().fft->execute2D(&f, 1);
        f.solvePoisson(cnfg->mass * pow(MVmodel.g_parameter, 2.0) * MVmodel.mu_parameter, MVmodel.g_parameter, ctx().mom);
        ctx().fft->execute2D(&f, 0);
        uf *= f;
    }
    store(uf, V_out);
}

/* `steps` momentum-space Langevin steps of main_optimized.cpp:243-269, 304
 * applied to V in place, with the configured coupling/kernel and `step`. */
void ref_evolve_momentum(double* V_io, int steps) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    fftw2D* fourier2 = ctx().fft;
    lfield<double, 9> uftmp(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 9> xi_local_x(cnfg->Nxl, cnfg->Nyl), xi_local_y(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 9> A_local(cnfg->Nxl, cnfg->Nyl), B_local(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 9> uxiulocal_x(cnfg->Nxl, cnfg->Nyl), uxiulocal_y(cnfg->Nxl, cnfg->Nyl);
    load(uftmp, V_io);
    for (int langevin = 0; langevin < steps; langevin++) {
        if (cnfg->CouplingChoice == NOISE_COUPLING_CONSTANT)
            generate_gaussian_with_noise_coupling_constant(&xi_local_x, &xi_local_y, ctx().mom, ctx().mpi, cnfg);
        else
            generate_gaussian(&xi_local_x, &xi_local_y, ctx().mpi, cnfg);
        fourier2->execute2D(&xi_local_x, 1);
        fourier2->execute2D(&xi_local_y, 1);
        prepare_A_local(&A_local, &xi_local_x, &xi_local_y, ctx().mom, ctx().mpi, cnfg->CouplingChoice, cnfg->KernelChoice);
        fourier2->execute2D(&A_local, 0);
        fourier2->execute2D(&xi_local_x, 0);
        fourier2->execute2D(&xi_local_y, 0);
        uxiulocal(&uxiulocal_x, &uxiulocal_y, &uftmp, &xi_local_x, &xi_local_y);
        fourier2->execute2D(&uxiulocal_x, 1);
        fourier2->execute2D(&uxiulocal_y, 1);
        prepare_A_local(&B_local, &uxiulocal_x, &uxiulocal_y, ctx().mom, ctx().mpi, cnfg->CouplingChoice, cnfg->KernelChoice);
        fourier2->execute2D(&B_local, 0);
        update_uf(&uftmp, &B_local, &A_local, cnfg->step);
    }
    store(uftmp, V_io);
}

/* Fixed coupling: the same step sequence with the reference's plain
 * generate_gaussian (field.h:2116) and prepare_A_local with
 * NOISE_COUPLING_CONSTANT (kernel factor 1, field.h:2035-2036, 2049-2050).
 * main_optimized.cpp:243-247 only reaches generate_gaussian for couplings other
 * than NOISE, so this composition of the reference's functions is how a fixed
 * coupling alpha_s (folded into `step`) is expressed. */
void ref_evolve_momentum_fixed(double* V_io, int steps) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    fftw2D* fourier2 = ctx().fft;
    lfield<double, 9> uftmp(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 9> xi_local_x(cnfg->Nxl, cnfg->Nyl), xi_local_y(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 9> A_local(cnfg->Nxl, cnfg->Nyl), B_local(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 9> uxiulocal_x(cnfg->Nxl, cnfg->Nyl), uxiulocal_y(cnfg->Nxl, cnfg->Nyl);
    load(uftmp, V_io);
    for (int langevin = 0; langevin < steps; langevin++) {
        generate_gaussian(&xi_local_x, &xi_local_y, ctx().mpi, cnfg);
        fourier2->execute2D(&xi_local_x, 1);
        fourier2->execute2D(&xi_local_y, 1);
        prepare_A_local(&A_local, &xi_local_x, &xi_local_y, ctx().mom, ctx().mpi, NOISE_COUPLING_CONSTANT, cnfg->KernelChoice);
        fourier2->execute2D(&A_local, 0);
        fourier2->execute2D(&xi_local_x, 0);
        fourier2->execute2D(&xi_local_y, 0);
        uxiulocal(&uxiulocal_x, &uxiulocal_y, &uftmp, &xi_local_x, &xi_local_y);
        fourier2->execute2D(&uxiulocal_x, 1);
        fourier2->execute2D(&uxiulocal_y, 1);
        prepare_A_local(&B_local, &uxiulocal_x, &uxiulocal_y, ctx().mom, ctx().mpi, NOISE_COUPLING_CONSTANT, cnfg->KernelChoice);
        fourier2->execute2D(&B_local, 0);
        update_uf(&uftmp, &B_local, &A_local, cnfg->step);
    }
    store(uftmp, V_io);
}

/* prepare_A_and_B_local (field.h:2368-2519) for every site, as the POSITION
 * branch of main_optimized.cpp:284-300 drives it (global xi and V gathered). */
void ref_prepare_A_and_B(double* A_out, double* B_out, const double* xi_x, const double* xi_y, const double* V,
                         int rr, int coupling, int kernel) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    gfield<double, 9> gx(Nx, Ny), gy(Nx, Ny), gv(Nx, Ny);
    memcpy((void*)gx.u, xi_x, sizeof(double) * 18 * Nx * Ny);
    memcpy((void*)gy.u, xi_y, sizeof(double) * 18 * Nx * Ny);
    memcpy((void*)gv.u, V, sizeof(double) * 18 * Nx * Ny);
    lfield<double, 9> A(cnfg->Nxl, cnfg->Nyl), B(cnfg->Nxl, cnfg->Nyl);
    A.setToZero();
    B.setToZero();
    for (int x = 0; x < cnfg->Nxl; x++)
        for (int y = 0; y < cnfg->Nyl; y++)
            prepare_A_and_B_local(x, y, x, y, &gx, &gy, &A, &B, &gv, ctx().pos, rr, (Coupling)coupling, (Kernel)kernel);
    store(A, A_out);
    store(B, B_out);
}

/* The correlated-noise set-up of main_optimized.cpp:145-157:
 * setCorrelationsForCouplingConstant, execute2D(-), allgather, decompose.
 * The factor is kept for ref_multiply_by_cholesky and copied to L_out
 * (V*V complex, row-major) when L_out is not null.  The matrix is zeroed
 * after allocation: the reference mallocs it uninitialised and reads the
 * whole of it in multiplyByCholesky (field.h:1653-1689); at the sizes it runs
 * (V*V*16 bytes, far above malloc's mmap threshold) those pages are zero. */
static gmatrix<double>* g_chol = nullptr;
void ref_cholesky_setup(double* L_out, double* corr_out) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    lfield<double, 1> corr(cnfg->Nxl, cnfg->Nyl);
    gfield<double, 1> corr_global(Nx, Ny);
    corr.setCorrelationsForCouplingConstant(ctx().mom);
    ctx().fft->execute2D(&corr, 0);
    corr_global.allgather(&corr, ctx().mpi);
    if (corr_out) memcpy(corr_out, (const void*)corr_global.u, sizeof(double) * 2 * Nx * Ny);
    if (g_chol) delete g_chol;
    g_chol = new gmatrix<double>(Nx * Ny, Nx * Ny);
    memset((void*)g_chol->u, 0, sizeof(double) * 2 * (size_t)Nx * Ny * Nx * Ny);
    g_chol->decompose(&corr_global);
    if (L_out) memcpy(L_out, (const void*)g_chol->u, sizeof(double) * 2 * (size_t)Nx * Ny * Nx * Ny);
}

/* gfield::multiplyByCholesky (field.h:1653-1689) with the set-up factor. */
void ref_multiply_by_cholesky(double* xi_io) {
    ensure_init(nullptr);
    gfield<double, 9> g(Nx, Ny);
    memcpy((void*)g.u, xi_io, sizeof(double) * 18 * Nx * Ny);
    g.multiplyByCholesky(g_chol);
    memcpy(xi_io, (const void*)g.u, sizeof(double) * 18 * Nx * Ny);
}

/* `steps` position-space steps of main_optimized.cpp:243-304 (POSITION
 * branch): generate_gaussian, allgather, multiplyByCholesky when the coupling
 * is NOISE (needs ref_cholesky_setup first), prepare_A_and_B_local at every
 * site with rr_hatta = rr, update_uf. */
void ref_evolve_position(double* V_io, int steps, int rr) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    lfield<double, 9> uftmp(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 9> xi_local_x(cnfg->Nxl, cnfg->Nyl), xi_local_y(cnfg->Nxl, cnfg->Nyl);
    gfield<double, 9> xi_global_x(Nx, Ny), xi_global_y(Nx, Ny), uf_global(Nx, Ny);
    lfield<double, 9> A_local(cnfg->Nxl, cnfg->Nyl), B_local(cnfg->Nxl, cnfg->Nyl);
    load(uftmp, V_io);
    for (int langevin = 0; langevin < steps; langevin++) {
        generate_gaussian(&xi_local_x, &xi_local_y, ctx().mpi, cnfg);
        xi_global_x.allgather(&xi_local_x, ctx().mpi);
        xi_global_y.allgather(&xi_local_y, ctx().mpi);
        if (cnfg->CouplingChoice == NOISE_COUPLING_CONSTANT) {
            xi_global_x.multiplyByCholesky(g_chol);
            xi_global_y.multiplyByCholesky(g_chol);
        }
        uf_global.allgather(&uftmp, ctx().mpi);
        A_local.setToZero();
        B_local.setToZero();
        for (int x = 0; x < cnfg->Nxl; x++)
            for (int y = 0; y < cnfg->Nyl; y++)
                prepare_A_and_B_local(x, y, x + ctx().mpi->getPosX() * cnfg->Nxl, y + ctx().mpi->getPosY() * cnfg->Nyl,
                                      &xi_global_x, &xi_global_y, &A_local, &B_local, &uf_global, ctx().pos, rr,
                                      cnfg->CouplingChoice, cnfg->KernelChoice);
        update_uf(&uftmp, &B_local, &A_local, cnfg->step);
    }
    store(uftmp, V_io);
}

/* gfield::reduce_hatta (field.h:1538-1567) after average_and_symmetrize of a
 * measurement of V (main_optimized.cpp:321-332). */
void ref_measure_hatta(const double* V, double* sum_io, double* err_io, int xr, int yr) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    lfield<double, 9> uf_copy(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 1> corr(cnfg->Nxl, cnfg->Nyl);
    gfield<double, 1> corr_global(Nx, Ny);
    lfield<double, 1> sum(cnfg->Nxl, cnfg->Nyl), err(cnfg->Nxl, cnfg->Nyl);
    load(uf_copy, V);
    load(sum, sum_io);
    load(err, err_io);
    ctx().fft->execute2D(&uf_copy, 1);
    uf_copy.trace(&corr);
    corr_global.allgather(&corr, ctx().mpi);
    corr_global.average_and_symmetrize();
    corr_global.reduce_hatta(&sum, &err, ctx().mpi, xr, yr);
    store(sum, sum_io);
    store(err, err_io);
}

/* One dipole measurement, main_optimized.cpp:321-334:
 * uf_copy = V; execute2D(+); trace; allgather; average_and_symmetrize;
 * reduce into sum/err (N*N complex each, accumulated in place).
 * corr_out (N*N complex) receives the symmetrised correlator. */
void ref_measure(const double* V, double* corr_out, double* sum_io, double* err_io) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    lfield<double, 9> uf_copy(cnfg->Nxl, cnfg->Nyl);
    lfield<double, 1> corr(cnfg->Nxl, cnfg->Nyl);
    gfield<double, 1> corr_global(Nx, Ny);
    lfield<double, 1> sum(cnfg->Nxl, cnfg->Nyl), err(cnfg->Nxl, cnfg->Nyl);
    load(uf_copy, V);
    load(sum, sum_io);
    load(err, err_io);
    ctx().fft->execute2D(&uf_copy, 1);
    uf_copy.trace(&corr);
    corr_global.allgather(&corr, ctx().mpi);
    corr_global.average_and_symmetrize();
    corr_global.reduce(&sum, &err, ctx().mpi);
    memcpy(corr_out, (const void*)corr_global.u, sizeof(double) * 2 * Nx * Ny);
    store(sum, sum_io);
    store(err, err_io);
}

/* print (field.h:2521-2547): appends the output table for one measurement to
 * <fileroot>_<Nx>_<Ny>_mpi1_r0.dat with x = 1/3/stat. */
void ref_print(int measurement, const double* sum_in, const double* err_in, double x, const char* fileroot) {
    ensure_init(nullptr);
    config* cnfg = ctx().cnfg;
    lfield<double, 1> sum(cnfg->Nxl, cnfg->Nyl), err(cnfg->Nxl, cnfg->Nyl);
    load(sum, sum_in);
    load(err, err_in);
    print(measurement, &sum, &err, ctx().mom, x, ctx().mpi, std::string(fileroot));
}

}  // extern "C"
