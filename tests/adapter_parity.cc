/*
 * Test infrastructure: the reference's SPME and Lanczos tests
 * (tests/spme/testspme.cc:103-145 and tests/lanczos/testlanczos.cc:81-148 of
 * the reference project) with the GPU adapters MobSpmeGpu / BrwnLanczosGpu
 * (include/stokesdt_b200_adapters.hpp) in place of MobSpme / BrwnLanczos,
 * called only through the reference's MobBase / BrwnBase interfaces (plus
 * RealMulVector / RecipMulVector, which MobSpme also has outside MobBase).
 *
 * Compiled against the reference headers (gnu++98, as the reference) by
 * tests/test_adapters.py and __graft_entry__.build() into tests/_bin/.
 *
 *   adapter_parity <in.bin> <out.bin>
 *
 * in.bin:  int32 npos, nrhs, dim, porder; double box, xi, rmax, alpha, beta,
 *          tol; pos[3N], rdi[N], f[nrhs][3N], z[nrhs][3N]
 * out.bin: v_full, v_real, v_recip [nrhs][3N] (v := alpha M f + beta f, as
 *          testspme.cc starts v from f), y1[3N] (1 RHS), y[nrhs][3N] (nrhs
 *          RHS) of BrwnLanczosGpu::Compute (max_iters 100, max_nrhs 16),
 *          v_ewald [nrhs][3N] from MobEwaldGpu (tol 1e-12, default xi) as
 *          testspme.cc's MobEwald
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "stokesdt_b200_adapters.hpp"

using stokesdt::BrwnBase;
using stokesdt::BrwnLanczosGpu;
using stokesdt::MobEwaldGpu;
using stokesdt::MobBase;
using stokesdt::MobSpmeGpu;

static bool read_all(FILE *fp, void *p, size_t bytes) { return fread(p, 1, bytes, fp) == bytes; }

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE *fi = fopen(argv[1], "rb");
    if (!fi) return 2;
    int hdr[4];
    double par[6];
    if (!read_all(fi, hdr, sizeof(hdr)) || !read_all(fi, par, sizeof(par))) return 2;
    const int npos = hdr[0], nrhs = hdr[1], dim = hdr[2], porder = hdr[3];
    const double box = par[0], xi = par[1], rmax = par[2], alpha = par[3], beta = par[4], tol = par[5];
    const int nm = 3 * npos, ldm = nm;
    std::vector<double> pos(nm), rdi(npos), f((size_t)ldm * nrhs), z((size_t)ldm * nrhs);
    if (!read_all(fi, &pos[0], sizeof(double) * nm) || !read_all(fi, &rdi[0], sizeof(double) * npos) ||
        !read_all(fi, &f[0], sizeof(double) * f.size()) || !read_all(fi, &z[0], sizeof(double) * z.size()))
        return 2;
    fclose(fi);

    // testspme.cc:118-133: construct, Init, Update, v starts as f, MulVector
    MobSpmeGpu *spme = new MobSpmeGpu(npos, &rdi[0], box, xi, rmax, dim, porder);
    MobBase *mob = spme;
    if (!mob->Init()) {
        fprintf(stderr, "MobSpmeGpu::Init failed\n");
        return 1;
    }
    mob->Update(&pos[0], &rdi[0]);
    if (mob->dim() != nm) return 1;
    std::vector<double> v_full(f), v_real(f), v_recip(f);
    mob->MulVector(nrhs, alpha, ldm, &f[0], beta, ldm, &v_full[0]);
    spme->RealMulVector(nrhs, alpha, ldm, &f[0], beta, ldm, &v_real[0]);
    spme->RecipMulVector(nrhs, alpha, ldm, &f[0], beta, ldm, &v_recip[0]);

    // testlanczos.cc:104-148: BrwnLanczos(nm, 100, 16, tol), 1 then nrhs RHS
    BrwnBase *brwn = new BrwnLanczosGpu(nm, 100, 16, tol);
    if (!brwn->Init()) {
        fprintf(stderr, "BrwnLanczosGpu::Init failed\n");
        return 1;
    }
    std::vector<double> y1(ldm, 0.0), y((size_t)ldm * nrhs, 0.0);
    brwn->Compute(mob, 1, ldm, &z[0], ldm, &y1[0]);
    brwn->Compute(mob, nrhs, ldm, &z[0], ldm, &y[0]);

    // testspme.cc:110-113, 127: the dense Ewald product through MobBase
    MobEwaldGpu *ewald = new MobEwaldGpu(npos, &rdi[0], box, 1.0e-12);
    MobBase *mob_ewald = ewald;
    if (!mob_ewald->Init()) {
        fprintf(stderr, "MobEwaldGpu::Init failed\n");
        return 1;
    }
    mob_ewald->Update(&pos[0], &rdi[0]);
    std::vector<double> v_ewald(f);
    mob_ewald->MulVector(nrhs, alpha, ldm, &f[0], beta, ldm, &v_ewald[0]);

    FILE *fo = fopen(argv[2], "wb");
    if (!fo) return 2;
    fwrite(&v_full[0], sizeof(double), v_full.size(), fo);
    fwrite(&v_real[0], sizeof(double), v_real.size(), fo);
    fwrite(&v_recip[0], sizeof(double), v_recip.size(), fo);
    fwrite(&y1[0], sizeof(double), y1.size(), fo);
    fwrite(&y[0], sizeof(double), y.size(), fo);
    fwrite(&v_ewald[0], sizeof(double), v_ewald.size(), fo);
    fclose(fo);
    delete ewald;
    delete brwn;
    delete spme;
    return 0;
}
