/*
 * stokesdt_b200_adapters.hpp -- header-only C++ adapters that put the B200
 * path behind the reference's own virtual interfaces, so BDSimBox, the mex
 * wrappers and the reference tests switch to the GPU by constructing a
 * different class.  Compile inside the reference tree (C++98 / gnu++98 like
 * the rest of it) with its src/mob and src/brwn include paths and link
 * libstokesdt_b200.so.
 *
 *   MobSpmeGpu     : MobBase   replaces MobSpme      (src/mob/mob_spme.h:21-125)
 *   MobEwaldGpu    : MobBase   replaces MobEwald     (src/mob/mob_ewald.h)
 *   BrwnLanczosGpu : BrwnBase  replaces BrwnLanczos  (src/brwn/brwn_lanczos.h:20-110)
 *   StericForceGpu : ForceBase replaces StericForce  (src/force/force_steric.h:20-86);
 *                    defined when force_base.h has been included first (the
 *                    reference's src/force on the include path)
 *
 * Error behaviour follows the reference: Init() returns false on bad
 * arguments or allocation failure; Update/MulVector/Compute return void and
 * report failures on stderr (the reference cannot fail there);
 * Lanczos non-convergence is reported, not fatal.
 */
#ifndef STOKESDT_B200_ADAPTERS_HPP_
#define STOKESDT_B200_ADAPTERS_HPP_

#include <cstdio>
#include <vector>

#include "brwn_base.h"
#include "mob_base.h"
#include "stokesdt_b200.h"

namespace stokesdt {

class MobSpmeGpu : public MobBase {
  public:
    MobSpmeGpu(const int npos, const double *rdi, const double box_size, const double xi,
               const double rmax, const int dim, const int porder, const int device = 0)
        : npos_(npos), rdi_(rdi, rdi + npos), box_size_(box_size), xi_(xi), rmax_(rmax),
          dim_(dim), porder_(porder), device_(device), h_(0)
    {
    }

    virtual ~MobSpmeGpu() { sdt_spme_destroy(h_); }

    virtual bool Init()
    {
        if (npos_ <= 0) return false;
        return sdt_spme_create(npos_, &rdi_[0], box_size_, xi_, rmax_, dim_, porder_, device_,
                               &h_) == SDT_OK;
    }

    virtual void Update(const double *pos, const double * /*rdi: fixed at construction*/)
    {
        Report(sdt_spme_update(h_, pos), "Update");
    }

    virtual void MulVector(const int num_rhs, const double alpha, const int ldf, const double *f,
                           const double beta, const int ldv, double *v)
    {
        Report(sdt_spme_mulvec(h_, SDT_MOB_FULL, num_rhs, alpha, ldf, f, beta, ldv, v), "MulVector");
    }

    void RealMulVector(const int num_rhs, const double alpha, const int ldf, const double *f,
                       const double beta, const int ldv, double *v)
    {
        Report(sdt_spme_mulvec(h_, SDT_MOB_REAL, num_rhs, alpha, ldf, f, beta, ldv, v),
               "RealMulVector");
    }

    void RecipMulVector(const int num_rhs, const double alpha, const int ldf, const double *f,
                        const double beta, const int ldv, double *v)
    {
        Report(sdt_spme_mulvec(h_, SDT_MOB_RECIP, num_rhs, alpha, ldf, f, beta, ldv, v),
               "RecipMulVector");
    }

    virtual int dim() { return 3 * npos_; }

    sdt_spme *handle() { return h_; }

  private:
    void Report(int st, const char *what)
    {
        if (st != SDT_OK)
            fprintf(stderr, "ERROR: MobSpmeGpu::%s: status %d: %s\n", what, st,
                    h_ ? sdt_spme_last_error(h_) : "not initialised");
    }

    MobSpmeGpu(const MobSpmeGpu &);
    void operator=(const MobSpmeGpu &);

    int npos_;
    std::vector<double> rdi_;
    double box_size_, xi_, rmax_;
    int dim_, porder_, device_;
    sdt_spme *h_;
};

class MobEwaldGpu : public MobBase {
  public:
    MobEwaldGpu(const int npos, const double *rdi, const double box_size, const double tol, const double xi = 0.0,
                const int device = 0)
        : npos_(npos), rdi_(rdi, rdi + npos), box_size_(box_size), tol_(tol), xi_(xi), device_(device), h_(0)
    {
    }

    virtual ~MobEwaldGpu() { sdt_ewald_destroy(h_); }

    virtual bool Init()
    {
        if (npos_ <= 0) return false;
        return sdt_ewald_create(npos_, &rdi_[0], box_size_, tol_, xi_, device_, &h_) == SDT_OK;
    }

    virtual void Update(const double *pos, const double * /*rdi: fixed at construction*/)
    {
        Report(sdt_ewald_update(h_, pos), "Update");
    }

    virtual void MulVector(const int num_rhs, const double alpha, const int ldf, const double *f,
                           const double beta, const int ldv, double *v)
    {
        Report(sdt_ewald_mulvec(h_, num_rhs, alpha, ldf, f, beta, ldv, v), "MulVector");
    }

    void GetMatrix(const int ldm, double *mat) { Report(sdt_ewald_get_matrix(h_, ldm, mat), "GetMatrix"); }

    virtual int dim() { return 3 * npos_; }

    sdt_ewald *handle() { return h_; }

  private:
    void Report(int st, const char *what)
    {
        if (st != SDT_OK)
            fprintf(stderr, "ERROR: MobEwaldGpu::%s: status %d: %s\n", what, st,
                    h_ ? sdt_ewald_last_error(h_) : "not initialised");
    }

    MobEwaldGpu(const MobEwaldGpu &);
    void operator=(const MobEwaldGpu &);

    int npos_;
    std::vector<double> rdi_;
    double box_size_, tol_, xi_;
    int device_;
    sdt_ewald *h_;
};

class BrwnLanczosGpu : public BrwnBase {
  public:
    BrwnLanczosGpu(const int dim, const int max_iters, const int max_nrhs, const double tol,
                   const int device = 0)
        : dim_(dim), max_iters_(max_iters), max_nrhs_(max_nrhs), tol_(tol), device_(device), h_(0)
    {
    }

    virtual ~BrwnLanczosGpu() { sdt_lanczos_destroy(h_); }

    virtual bool Init()
    {
        return sdt_lanczos_create(dim_, max_iters_, max_nrhs_, tol_, device_, &h_) == SDT_OK;
    }

    /* mob must be a MobSpmeGpu or a MobEwaldGpu (the products run on its
     * GPU engine). */
    virtual void Compute(MobBase *mob, const int num_rhs, const int ldz, const double *z,
                         const int ldy, double *y)
    {
        MobSpmeGpu *g = dynamic_cast<MobSpmeGpu *>(mob);
        MobEwaldGpu *ew = dynamic_cast<MobEwaldGpu *>(mob);
        if (g == 0 && ew == 0) {
            fprintf(stderr, "ERROR: BrwnLanczosGpu::Compute needs a MobSpmeGpu or a MobEwaldGpu\n");
            return;
        }
        int groups = (num_rhs + max_nrhs_ - 1) / max_nrhs_;
        std::vector<int> iters(groups > 0 ? groups : 1, 0);
        const int st = g ? sdt_lanczos_compute(h_, g->handle(), num_rhs, ldz, z, ldy, y, &iters[0])
                         : sdt_lanczos_compute_ewald(h_, ew->handle(), num_rhs, ldz, z, ldy, y, &iters[0]);
        if (st == SDT_ERR_NOT_CONVERGED)
            fprintf(stderr, "WARNING: BrwnLanczosGpu: NOT converged\n");
        else if (st != SDT_OK)
            fprintf(stderr, "ERROR: BrwnLanczosGpu::Compute: status %d: %s\n", st,
                    sdt_lanczos_last_error(h_));
    }

  private:
    BrwnLanczosGpu(const BrwnLanczosGpu &);
    void operator=(const BrwnLanczosGpu &);

    int dim_, max_iters_, max_nrhs_;
    double tol_;
    int device_;
    sdt_lanczos *h_;
};

#ifdef FORCE_BASE_H_
class StericForceGpu : public ForceBase {
  public:
    StericForceGpu(const int npos, const double *rdi, const double box_size, const double steric_r0,
                   const double steric_k0, const int device = 0)
        : ForceBase(npos), rdi_(rdi, rdi + npos), box_size_(box_size), r0_(steric_r0),
          k0_(steric_k0), device_(device), h_(0)
    {
    }

    virtual ~StericForceGpu() { sdt_steric_destroy(h_); }

    virtual bool Init()
    {
        return sdt_steric_create((int)rdi_.size(), &rdi_[0], box_size_, r0_, k0_, device_, &h_) ==
               SDT_OK;
    }

    virtual void Accumulate(const double *pos, const double * /*rdi: fixed at construction*/,
                            double *f)
    {
        const int st = sdt_steric_accumulate(h_, pos, f);
        if (st != SDT_OK)
            fprintf(stderr, "ERROR: StericForceGpu::Accumulate: status %d: %s\n", st,
                    h_ ? sdt_steric_last_error(h_) : "not initialised");
    }

  private:
    StericForceGpu(const StericForceGpu &);
    void operator=(const StericForceGpu &);

    std::vector<double> rdi_;
    double box_size_, r0_, k0_;
    int device_;
    sdt_steric *h_;
};
#endif  // FORCE_BASE_H_

}  // namespace stokesdt

#endif  // STOKESDT_B200_ADAPTERS_HPP_
