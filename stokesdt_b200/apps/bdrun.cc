// bdrun: Brownian dynamics on the B200 path with the command line and input
// files of the reference's driver (bin/main/main.cc, BDSimBox
// src/simbox/simbox_bd.cc:89-366):
//
//   bdrun --config run.cfg --model run.mod --xyz start.xyz -n NSTEPS
//
// Config keys (defaults as BDSimBox): delta-t 0.001, mob-method
// (ewald | ewald-gpu | spme | spme-gpu; default ewald), ewald-tol 1e-4,
// brownian-method (lanczos | lanczos-gpu), mob-interval 100,
// spme-nfft-grids 128, spme-porder 4, spme-xi 0.5, spme-rmax 4.0,
// lanczos-maxiters 50, lanczos-maxnrhs 20, lanczos-tol 1e-3, traj-startstep
// 0, traj-interval -1, traj-output trajectory.xyz, random-seed 1234.
// The model file's par lines give the radii, its steric line the steric
// force.  Positions, forces and random vectors stay on the GPU (the dense
// Ewald matrix too: 72 N^2 bytes); frames are written in the reference's
// XYZ layout.  The reference's Cholesky and random Brownian methods are not
// offered (not on the GPU path).
#include <getopt.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "stokesdt_b200.h"

namespace {

std::string cfg_str(const char *cfg, const char *key, const char *def)
{
    char buf[512];
    const int st = sdt_config_get(cfg, key, buf, sizeof(buf));
    if (st < 0) {
        std::fprintf(stderr, "cannot read %s (or key %s is duplicated)\n", cfg, key);
        std::exit(1);
    }
    return st == 0 ? std::string(buf) : std::string(def);
}

double cfg_f(const char *cfg, const char *key, double def)
{
    return std::atof(cfg_str(cfg, key, std::to_string(def).c_str()).c_str());
}

int cfg_i(const char *cfg, const char *key, int def)
{
    return std::atoi(cfg_str(cfg, key, std::to_string(def).c_str()).c_str());
}

void usage(const char *call)
{
    std::fprintf(stderr,
                 "Usage: %s --config FILE --model FILE --xyz FILE [-n NSTEPS] [--device N]\n"
                 "  mob-method spme|spme-gpu, brownian-method lanczos|lanczos-gpu\n",
                 call);
}

}  // namespace

int main(int argc, char **argv)
{
    const struct option opts[] = {{"help", 0, nullptr, 'h'},   {"nsteps", 1, nullptr, 'n'},
                                  {"config", 1, nullptr, 10},  {"model", 1, nullptr, 20},
                                  {"xyz", 1, nullptr, 30},     {"device", 1, nullptr, 40},
                                  {nullptr, 0, nullptr, 0}};
    const char *cfg = nullptr, *model = nullptr, *xyz = nullptr;
    int nsteps = 1, device = 0, c;
    while ((c = getopt_long(argc, argv, ":hn:", opts, nullptr)) != -1) {
        switch (c) {
            case 'h': usage(argv[0]); return 0;
            case 'n': nsteps = std::atoi(optarg); break;
            case 10: cfg = optarg; break;
            case 20: model = optarg; break;
            case 30: xyz = optarg; break;
            case 40: device = std::atoi(optarg); break;
            default: usage(argv[0]); return 1;
        }
    }
    if (!cfg || !model || !xyz || nsteps <= 0) {
        usage(argv[0]);
        return 1;
    }
    const std::string mob_method = cfg_str(cfg, "mob-method", "ewald");
    const std::string brwn_method = cfg_str(cfg, "brownian-method", "cholesky");
    const bool ewald = mob_method == "ewald" || mob_method == "ewald-gpu";
    if (!ewald && mob_method != "spme" && mob_method != "spme-gpu") {
        std::fprintf(stderr, "mob-method %s: only ewald / spme (and their -gpu names) run on the GPU path\n",
                     mob_method.c_str());
        return 1;
    }
    if (brwn_method != "lanczos" && brwn_method != "lanczos-gpu") {
        std::fprintf(stderr, "brownian-method %s: only lanczos / lanczos-gpu run on the GPU path\n",
                     brwn_method.c_str());
        return 1;
    }
    const double dt = cfg_f(cfg, "delta-t", 0.001);
    const int mob_interval = cfg_i(cfg, "mob-interval", 100);
    const int K = cfg_i(cfg, "spme-nfft-grids", 128);
    const int porder = cfg_i(cfg, "spme-porder", 4);
    const double xi = cfg_f(cfg, "spme-xi", 0.5);
    const double rmax = cfg_f(cfg, "spme-rmax", 4.0);
    const int max_iters = cfg_i(cfg, "lanczos-maxiters", 50);
    const int max_nrhs = cfg_i(cfg, "lanczos-maxnrhs", 20);
    const double tol = cfg_f(cfg, "lanczos-tol", 1.0e-3);
    const int traj_start = cfg_i(cfg, "traj-startstep", 0);
    const int traj_interval = cfg_i(cfg, "traj-interval", -1);
    const std::string traj_out = cfg_str(cfg, "traj-output", "trajectory.xyz");
    const unsigned long long seed = std::strtoull(cfg_str(cfg, "random-seed", "1234").c_str(), nullptr, 10);

    int npos = 0;
    if (sdt_xyz_count(xyz, &npos) != 0) {
        std::fprintf(stderr, "cannot read %s\n", xyz);
        return 1;
    }
    std::vector<double> pos(3 * (size_t)npos), rdi(npos);
    double box[3];
    int start_step = 0;
    double start_time = 0.0;
    if (sdt_xyz_read(xyz, model, npos, pos.data(), rdi.data(), box, &start_step, &start_time) != 0) {
        std::fprintf(stderr, "malformed XYZ file %s\n", xyz);
        return 1;
    }
    // cubic boxes only; the reference's writer prints Lx with 6 significant
    // digits and Ly, Lz with 10 (molecule_io.cc:396-397), so compare at that
    // precision and take the precise edge
    if (std::fabs(box[0] - box[2]) > 1e-5 * box[2] || std::fabs(box[1] - box[2]) > 1e-9 * box[2]) {
        std::fprintf(stderr, "only cubic boxes are supported (Lx = Ly = Lz)\n");
        return 1;
    }
    box[0] = box[1] = box[2];
    double r0 = 0.0, k0 = 0.0;
    const int has_steric = sdt_model_steric(model, &r0, &k0) == 0;

    sdt_spme *mob = nullptr;
    sdt_ewald *ew = nullptr;
    sdt_lanczos *lz = nullptr;
    sdt_steric *st = nullptr;
    sdt_bd *bd = nullptr;
    const double ewald_tol = cfg_f(cfg, "ewald-tol", 1e-4);
    int rc = ewald ? sdt_ewald_create(npos, rdi.data(), box[0], ewald_tol, 0.0, device, &ew)
                   : sdt_spme_create(npos, rdi.data(), box[0], xi, rmax, K, porder, device, &mob);
    if (rc != SDT_OK) {
        std::fprintf(stderr, "%s set-up failed (status %d): check the %s keys\n", ewald ? "Ewald" : "SPME", rc,
                     ewald ? "ewald-*" : "spme-*");
        return 1;
    }
    rc = sdt_lanczos_create(3 * npos, max_iters, max_nrhs, tol, device, &lz);
    if (rc == SDT_OK && has_steric) rc = sdt_steric_create(npos, rdi.data(), box[0], r0, k0, device, &st);
    if (rc == SDT_OK)
        rc = ewald ? sdt_bd_create_ewald(ew, lz, st, dt, mob_interval, seed, &bd)
                   : sdt_bd_create(mob, lz, st, dt, mob_interval, seed, &bd);
    if (rc == SDT_OK) rc = sdt_bd_set_positions(bd, pos.data());
    if (rc == SDT_OK) rc = sdt_bd_set_step(bd, start_step);
    if (rc != SDT_OK) {
        std::fprintf(stderr, "set-up failed (status %d)\n", rc);
        return 1;
    }
    if (ewald)
        std::printf("bdrun: %d particles, box %g, dense Ewald (tol %g), dt %g, mob-interval %d, steric %s\n", npos,
                    box[0], ewald_tol, dt, mob_interval, has_steric ? "on" : "off");
    else
        std::printf("bdrun: %d particles, box %g, K %d, p %d, xi %g, rmax %g, dt %g, mob-interval %d, steric %s\n",
                    npos, box[0], K, porder, xi, rmax, dt, mob_interval, has_steric ? "on" : "off");
    const auto t0 = std::chrono::steady_clock::now();
    long long istep = start_step;
    double time = start_time;
    for (int k = 0; k < nsteps && rc == SDT_OK; k++) {
        rc = sdt_bd_advance(bd, 1);
        istep++;
        time += dt;
        if (rc == SDT_OK && traj_interval > 0 && istep > traj_start && istep % traj_interval == 0) {
            rc = sdt_bd_get_positions(bd, pos.data());
            if (rc == SDT_OK &&
                sdt_xyz_write(traj_out.c_str(), 1, npos, box, (int)istep, time, pos.data()) != 0) {
                std::fprintf(stderr, "cannot write %s\n", traj_out.c_str());
                rc = SDT_ERR_INVALID;
            }
        }
    }
    if (rc == SDT_OK) rc = sdt_bd_get_positions(bd, pos.data());
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    long long nc = 0;
    sdt_bd_info(bd, nullptr, &nc, nullptr);
    if (rc != SDT_OK) std::fprintf(stderr, "failed at step %lld: %s\n", istep, sdt_bd_last_error(bd));
    std::printf("bdrun: %d steps in %.3f s (%.2f steps/s), Lanczos calls over tol: %lld\n", nsteps, secs,
                nsteps / secs, nc);
    sdt_bd_destroy(bd);
    sdt_steric_destroy(st);
    sdt_lanczos_destroy(lz);
    sdt_spme_destroy(mob);
    sdt_ewald_destroy(ew);
    return rc == SDT_OK ? 0 : 1;
}
