// jw_config.cpp -- the reference's run-configuration file and output table,
// on the host: config::read_config_from_file (config.h:76-136) and
// print (field.h:2521-2547).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/jimwlk.h"

#define JW_EXPORT extern "C" __attribute__((visibility("default")))

JW_EXPORT jw_status jw_config_defaults(jw_config* c) {
    if (!c) return JW_EINVAL;
    std::memset(c, 0, sizeof(*c));
    c->Nx = 64;
    c->Ny = 64;
    c->stat = 4;
    c->mu = 30.72;
    c->mass = 0.0001;
    c->elementaryWilsonLines = 50;
    std::strcpy(c->file_name, "output");
    c->langevin_steps = 100;
    c->measurements = 100;
    c->step = 0.0004;
    c->EvolutionChoice = JW_MOMENTUM_EVOLUTION;
    c->CouplingChoice = JW_NOISE_COUPLING_CONSTANT;
    c->KernelChoice = JW_SIN_KERNEL;
    c->seed = 1;
    return JW_OK;
}

// Same fscanf sequence as config.h:83-101; mu, mass and step pass through a
// float as in the reference.  A missing file is an error (the reference would
// crash on a null FILE*).
JW_EXPORT jw_status jw_config_read(jw_config* c, const char* path) {
    if (!c || !path) return JW_EINVAL;
    FILE* f = std::fopen(path, "r");
    if (!f) return JW_EINVAL;
    float tmp;
    char name[64] = {0};
    char evolution[100] = {0}, coupling[100] = {0}, kernel[100] = {0};
    int ok = 1;
    ok &= std::fscanf(f, "stat = %i\n", &c->stat) == 1;
    if (std::fscanf(f, "mu = %f\n", &tmp) == 1) c->mu = tmp; else ok = 0;
    if (std::fscanf(f, "mass = %f\n", &tmp) == 1) c->mass = tmp; else ok = 0;
    ok &= std::fscanf(f, "elementaryWilsonLines = %i\n", &c->elementaryWilsonLines) == 1;
    if (std::fscanf(f, "file_name = %63s\n", name) == 1) std::strcpy(c->file_name, name); else ok = 0;
    ok &= std::fscanf(f, "langevin_steps = %i\n", &c->langevin_steps) == 1;
    ok &= std::fscanf(f, "measurements = %i\n", &c->measurements) == 1;
    if (std::fscanf(f, "step = %f\n", &tmp) == 1) c->step = tmp; else ok = 0;
    if (std::fscanf(f, "EvolutionChoice = %99s\n", evolution) != 1) evolution[0] = 0;
    if (std::fscanf(f, "CouplingChoice = %99s\n", coupling) != 1) coupling[0] = 0;
    if (std::fscanf(f, "KernelChoice = %99s\n", kernel) != 1) kernel[0] = 0;
    std::fclose(f);
    if (!std::strcmp(evolution, "MOMENTUM_EVOLUTION")) c->EvolutionChoice = JW_MOMENTUM_EVOLUTION;
    if (!std::strcmp(evolution, "POSITION_EVOLUTION")) c->EvolutionChoice = JW_POSITION_EVOLUTION;
    if (!std::strcmp(coupling, "SQRT_COUPLING_CONSTANT")) c->CouplingChoice = JW_SQRT_COUPLING_CONSTANT;
    if (!std::strcmp(coupling, "NOISE_COUPLING_CONSTANT")) c->CouplingChoice = JW_NOISE_COUPLING_CONSTANT;
    if (!std::strcmp(coupling, "HATTA_COUPLING_CONSTANT")) c->CouplingChoice = JW_HATTA_COUPLING_CONSTANT;
    // this library's fixed coupling (no reference spelling exists)
    if (!std::strcmp(coupling, "FIXED_COUPLING_CONSTANT")) c->CouplingChoice = JW_FIXED_COUPLING_CONSTANT;
    if (!std::strcmp(kernel, "LINEAR_KERNEL")) c->KernelChoice = JW_LINEAR_KERNEL;
    if (!std::strcmp(kernel, "SIN_KERNEL")) c->KernelChoice = JW_SIN_KERNEL;
    return ok ? JW_OK : JW_EINVAL;
}

// print (field.h:2521-2547): one line per momentum with |kx - ky| <= 4:
// "meas kx ky \t |phat| x*phat2*Re(sum) x*phat2*Re(err)".
extern "C" jw_status jw_print_host(int N, int measurement, const double* sum, const double* err, double x,
                                   const char* fileroot) {
    char filename[512];
    std::snprintf(filename, sizeof filename, "%s_%i_%i_mpi%i_r%i.dat", fileroot, N, N, 1, 0);
    FILE* f = std::fopen(filename, "a+");
    if (!f) return JW_EINVAL;
    for (int xx = 0; xx < N; ++xx)
        for (int yy = 0; yy < N; ++yy) {
            const long i = (long)xx * N + yy;
            if (std::fabs((double)(xx - yy)) <= 4) {
                const double sx = std::sin(M_PI * xx / (1.0 * N)), sy = std::sin(M_PI * yy / (1.0 * N));
                const double ph2 = 4.0 * std::pow(sx, 2.0) + 4.0 * std::pow(sy, 2.0);
                std::fprintf(f, "%i %i %i \t %f %e %e\n", measurement, xx, yy, std::sqrt(ph2), x * ph2 * sum[2 * i],
                             x * ph2 * err[2 * i]);
            }
        }
    std::fclose(f);
    return JW_OK;
}
