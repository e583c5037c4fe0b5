// jimwlk_main.cpp -- main_optimized.cpp on one GPU: the same configuration
// file, the same sequence (statistics -> MV initial condition -> [Hatta loop
// over distances] -> Langevin steps -> measurements) and the same output
// table (output_optimized_<Nx>_<Ny>_mpi1_r0.dat), with the reference's
// progress lines.
//
//   jimwlk_main <px> <py> <config> [--N n] [--device d] [--seed s] [--call-for-call] [--mixed]
//
// <px> <py> are the reference's MPI grid arguments (ignored: one GPU holds the
// lattice).  --N sets the lattice side (the reference fixes it at compile
// time, 64 by default).  By default each Langevin step is one fused library
// call (jw_evolve_momentum / jw_evolve_position), and the Hatta branches
// (HATTA coupling, main_optimized.cpp:200-216) run together as events of the
// batched engine, one per (ix, iy), stepped in one launch sequence (FP64, or
// mixed precision with --mixed; at sizes that are not powers of two the
// branches run one after another).  --call-for-call runs the body of
// main_optimized.cpp:232-304 literally, one adapter call per reference call,
// branch after branch.  All modes draw the same noise: Langevin step n of the
// run (branches in the reference's order) uses stream index n, MV slice n
// stream index n.  Exit status 0 on success (the reference returns 1).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "jimwlk.hpp"

using namespace jimwlk;

namespace {

struct timer {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double seconds() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

// The Hatta branches of one statistics sample (main_optimized.cpp:200-216,
// 331-332) as events of the batched engine: branch b = (ix, iy) starts from
// the initial condition uf, evolves with rr = |(ix, iy)|^2 (wrapped) and noise
// indices from dev.noise_step + b * langevin_steps on, and adds its
// symmetrised correlator at (ix, iy) to sum[t], err[t] at each measurement.
void run_hatta_batched(device& dev, const config& cnfg, lfield<double, 9>& uf,
                       std::vector<std::unique_ptr<lfield<double, 1>>>& sum,
                       std::vector<std::unique_ptr<lfield<double, 1>>>& err, int device_id, bool mixed) {
    const int Nx = cnfg.Nx, Ny = cnfg.Ny, steps = cnfg.langevin_steps;
    struct Branch { int ix, iy, rr; };
    std::vector<Branch> br;
    for (int ix = 0; ix < Nx; ++ix)
        for (int iy = ix - 1; iy < ix + 2; ++iy) {
            if (iy < 0 || iy >= Ny) continue;
            double dix = ix, diy = iy;
            if (dix >= Nx / 2) dix -= Nx;
            if (dix < -Nx / 2) dix += Nx;
            if (diy >= Ny / 2) diy -= Ny;
            if (diy < -Ny / 2) diy += Ny;
            br.push_back({ix, iy, (int)(dix * dix + diy * diy)});
        }
    jw_engine_options o{};
    o.precision = mixed ? JW_PRECISION_MIXED : JW_PRECISION_FP64;
    jw_engine* e = nullptr;
    check(jw_engine_create(&o, device_id, &e), "jw_engine_create");
    struct Guard { jw_engine* e; ~Guard() { jw_engine_destroy(e); } } guard{e};
    const std::vector<std::complex<double>> V0 = uf.get();
    std::vector<int> ids(br.size()), xs(br.size()), ys(br.size());
    for (size_t b = 0; b < br.size(); ++b) {
        jw_event_desc d{};
        d.N = Nx;
        d.ny_slices = 0;
        d.mu = cnfg.mu;
        d.mass = cnfg.mass;
        d.step = cnfg.step;
        d.coupling = JW_HATTA_COUPLING_CONSTANT;
        d.kernel = cnfg.KernelChoice;
        d.seed = cnfg.seed;
        d.position_space = cnfg.EvolutionChoice == POSITION_EVOLUTION;
        d.rr = br[b].rr;
        d.step0 = dev.noise_step + (uint64_t)b * steps;
        check(jw_engine_add_event(e, &d, &ids[b]), "jw_engine_add_event");
        if (b == 0) check(jw_engine_set_V(e, ids[b], reinterpret_cast<const double*>(V0.data())), "jw_engine_set_V");
        else check(jw_engine_copy_V(e, ids[b], ids[0]), "jw_engine_copy_V");  // uftmp = uf
        xs[b] = br[b].ix;
        ys[b] = br[b].iy;
    }
    const int n = (int)ids.size();
    const int every = cnfg.langevin_steps / cnfg.measurements;
    std::vector<double> vs(n), ve(n);
    for (int langevin = 0; langevin < steps; ++langevin) {
        timer te;
        std::printf("Performing evolution step no. %i (%d Hatta branches)\n", langevin, n);
        check(jw_engine_step(e, ids.data(), n, 1), "jw_engine_step");
        check(jw_engine_sync(e), "jw_engine_sync");
        std::printf("Evolution time: %g\n", te.seconds());
        if (langevin % every == 0) {
            const int time = (int)(langevin * cnfg.measurements / cnfg.langevin_steps);
            check(jw_engine_measure(e, ids.data(), n), "jw_engine_measure");
            check(jw_engine_correlator_at(e, ids.data(), n, xs.data(), ys.data(), vs.data(), ve.data()),
                  "jw_engine_correlator_at");
            check(jw_engine_reset_correlators(e, ids.data(), n), "jw_engine_reset_correlators");
            // reduce_hatta (field.h:1538-1564): one site per branch
            std::vector<std::complex<double>> hs = sum[time]->get(), he = err[time]->get();
            for (int b = 0; b < n; ++b) {
                const long i = (long)xs[b] * Ny + ys[b];
                hs[i] += vs[b];
                he[i] += ve[b];
            }
            sum[time]->set(hs);
            err[time]->set(he);
        }
    }
    dev.noise_step += (uint64_t)n * steps;
}

int usage() {
    std::fprintf(stderr, "usage: jimwlk_main <px> <py> <config> [--N n] [--device d] [--seed s] [--call-for-call] "
                         "[--mixed]\n");
    return 2;
}

}  // namespace

int main(int argc, char* argv[]) {
    if (argc < 4) return usage();
    int N = 64, device_id = 0;
    bool call_for_call = false, seed_given = false, mixed = false;
    uint64_t seed = 1;
    for (int i = 4; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--N") && i + 1 < argc) N = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device_id = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--seed") && i + 1 < argc) {
            seed = std::strtoull(argv[++i], nullptr, 10);
            seed_given = true;
        } else if (!std::strcmp(argv[i], "--call-for-call")) call_for_call = true;
        else if (!std::strcmp(argv[i], "--mixed")) mixed = true;
        else return usage();
    }
    try {
        std::printf("INITIALIZATION\n");
        config cnfg(N);
        cnfg.read_config_from_file(argv[3]);
        if (seed_given) cnfg.seed = seed;
        if (cnfg.langevin_steps < 1 || cnfg.measurements < 1 || cnfg.langevin_steps / cnfg.measurements < 1) {
            std::fprintf(stderr, "jimwlk_main: need 1 <= measurements <= langevin_steps\n");
            return 2;
        }
        mpi_class mpi(argc, argv);
        mpi.mpi_init(&cnfg);
        mpi.mpi_exchange_grid();
        momenta momtable(&cnfg, &mpi);
        momtable.set();
        positions postable(&cnfg, &mpi);
        postable.set();
        device dev(cnfg, device_id);
        MV_class MVmodel(1.0, cnfg.mu / cnfg.Nx, cnfg.elementaryWilsonLines);
        fftw2D fourier2(dev);
        fourier2.init2D();

        std::printf("ALLOCATION\n");
        lfield<double, 9> f(dev), uf(dev), xi_local_x(dev), xi_local_y(dev), A_local(dev), B_local(dev), uftmp(dev);
        lfield<double, 9> uxiulocal_x(dev), uxiulocal_y(dev), uf_copy(dev);
        lfield<double, 1> zero(dev), corr(dev);
        // the reference allocates one accumulator per step (main_optimized.cpp:131-132);
        // only the first `measurements` are ever used
        std::vector<std::unique_ptr<lfield<double, 1>>> sum, err;
        for (int i = 0; i < cnfg.measurements; ++i) {
            sum.emplace_back(new lfield<double, 1>(zero));
            err.emplace_back(new lfield<double, 1>(zero));
        }

        const Evolution evo = cnfg.EvolutionChoice;
        const Coupling cp = cnfg.CouplingChoice;
        // fixed coupling: NOISE kernel factor 1 with plain noise
        const Coupling kernel_cp = cp == FIXED_COUPLING_CONSTANT ? NOISE_COUPLING_CONSTANT : cp;
        std::unique_ptr<gmatrix<double>> cholesky;
        if (evo == POSITION_EVOLUTION && cp == NOISE_COUPLING_CONSTANT) {  // :145-157
            corr.setCorrelationsForCouplingConstant(&momtable);
            fourier2.execute2D(&corr, 0);
            cholesky.reset(new gmatrix<double>(dev));
            cholesky->decompose(&corr);
            std::printf("cholesky decomposition finished\n");
        }
        const int Nx = cnfg.Nx, Ny = cnfg.Ny;
        const int every = cnfg.langevin_steps / cnfg.measurements;

        for (int stat = 0; stat < cnfg.stat; ++stat) {
            timer ts;
            std::printf("Gatherting stat sample no. %i\n", stat);
            timer ti;
            uf.setToUnit();
            for (int i = 0; i < MVmodel.Ny_parameter; ++i) {  // :180-191
                f.setMVModel(&MVmodel);
                fourier2.execute2D(&f, 1);
                f.solvePoisson(cnfg.mass * MVmodel.g_parameter * MVmodel.g_parameter * MVmodel.mu_parameter,
                               MVmodel.g_parameter, &momtable);
                fourier2.execute2D(&f, 0);
                uf *= f;
            }
            dev.sync();
            std::printf("Initial condition time: %g\n", ti.seconds());

            // the batched engine takes power-of-two lattices; other sizes run the branches one by one
            const bool engine_size = Nx >= 8 && Nx <= 2048 && (Nx & (Nx - 1)) == 0;
            if (cp == HATTA_COUPLING_CONSTANT && !call_for_call && engine_size) {
                run_hatta_batched(dev, cnfg, uf, sum, err, device_id, mixed);
                dev.sync();
                std::printf("Statistics time: %g\n", ts.seconds());
                continue;
            }
            const int upper_bound_x = cp == HATTA_COUPLING_CONSTANT ? Nx : 1;  // :200-216
            for (int ix = 0; ix < upper_bound_x; ++ix) {
                const int lower_bound_y = cp == HATTA_COUPLING_CONSTANT ? ix - 1 : 0;
                const int upper_bound_y = cp == HATTA_COUPLING_CONSTANT ? ix + 2 : 1;
                for (int iy = lower_bound_y; iy < upper_bound_y; ++iy) {
                    if (iy < 0 || iy >= Ny) continue;
                    double dix = ix, diy = iy;
                    if (dix >= Nx / 2) dix -= Nx;
                    if (dix < -Nx / 2) dix += Nx;
                    if (diy >= Ny / 2) diy -= Ny;
                    if (diy < -Ny / 2) diy += Ny;
                    const int rr_hatta = (int)(dix * dix + diy * diy);
                    uftmp = uf;
                    for (int langevin = 0; langevin < cnfg.langevin_steps; ++langevin) {
                        timer te;
                        std::printf("Performing evolution step no. %i\n", langevin);
                        if (!call_for_call) {
                            const uint64_t step_index = dev.noise_step++;
                            if (evo == MOMENTUM_EVOLUTION)
                                check(jw_evolve_momentum(dev.ctx, uftmp.f, step_index, 1), "jw_evolve_momentum");
                            else
                                check(jw_evolve_position(dev.ctx, uftmp.f, step_index, 1, rr_hatta,
                                                         cholesky ? cholesky->L : nullptr),
                                      "jw_evolve_position");
                        } else {
                            // :243-304, one adapter call per reference call
                            if (evo == MOMENTUM_EVOLUTION && cp == NOISE_COUPLING_CONSTANT)
                                generate_gaussian_with_noise_coupling_constant(&xi_local_x, &xi_local_y, &momtable,
                                                                               &mpi, &cnfg);
                            else
                                generate_gaussian(&xi_local_x, &xi_local_y, &mpi, &cnfg);
                            if (evo == MOMENTUM_EVOLUTION) {
                                fourier2.execute2D(&xi_local_x, 1);
                                fourier2.execute2D(&xi_local_y, 1);
                                prepare_A_local(&A_local, &xi_local_x, &xi_local_y, &momtable, &mpi, kernel_cp,
                                                cnfg.KernelChoice);
                                fourier2.execute2D(&A_local, 0);
                                fourier2.execute2D(&xi_local_x, 0);
                                fourier2.execute2D(&xi_local_y, 0);
                                uxiulocal(&uxiulocal_x, &uxiulocal_y, &uftmp, &xi_local_x, &xi_local_y);
                                fourier2.execute2D(&uxiulocal_x, 1);
                                fourier2.execute2D(&uxiulocal_y, 1);
                                prepare_A_local(&B_local, &uxiulocal_x, &uxiulocal_y, &momtable, &mpi, kernel_cp,
                                                cnfg.KernelChoice);
                                fourier2.execute2D(&B_local, 0);
                            } else {
                                // the gathers are identities on one GPU
                                if (cp == NOISE_COUPLING_CONSTANT) {
                                    xi_local_x.multiplyByCholesky(cholesky.get());
                                    xi_local_y.multiplyByCholesky(cholesky.get());
                                }
                                prepare_A_and_B(&xi_local_x, &xi_local_y, &A_local, &B_local, &uftmp, &postable,
                                                rr_hatta, cp, cnfg.KernelChoice);
                            }
                            update_uf(&uftmp, &B_local, &A_local, cnfg.step);
                        }
                        dev.sync();
                        std::printf("Evolution time: %g\n", te.seconds());

                        if (langevin % every == 0) {  // :314-336
                            const int time = (int)(langevin * cnfg.measurements / cnfg.langevin_steps);
                            uf_copy = uftmp;
                            fourier2.execute2D(&uf_copy, 1);
                            uf_copy.trace(&corr);
                            corr.average_and_symmetrize();
                            if (cp == HATTA_COUPLING_CONSTANT)
                                corr.reduce_hatta(sum[time].get(), err[time].get(), &mpi, ix, iy);
                            else
                                corr.reduce(sum[time].get(), err[time].get(), &mpi);
                        }
                    }
                }
            }
            dev.sync();
            std::printf("Statistics time: %g\n", ts.seconds());
        }
        const std::string file_name = "output_optimized";
        for (int i = cnfg.measurements - 1; i < cnfg.measurements; ++i)
            print(i, sum[i].get(), err[i].get(), &momtable, 1.0 / 3.0 / cnfg.stat, &mpi, file_name);
        dev.sync();
    } catch (const error& e) {
        std::fprintf(stderr, "jimwlk_main: %s\n", e.what());
        return 1;
    }
    return 0;
}
