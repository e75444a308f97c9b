// chswe.hpp -- C++ host mirror of the reference's operator_t / stvec_t /
// timescheme_t interfaces (src/operator_mod.f90:11-41, src/stvec/stvec_mod.f90:10-30,
// src/time_schemes/timescheme_mod.f90:9-24) over the C ABI in chswe.h.
// Header-only; errors throw std::runtime_error carrying swe_last_error().
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "chswe.h"

namespace chswe_host {

inline void check(int rc, const swe_ctx *ctx, const char *what)
{
    if (rc != SWE_OK)
        throw std::runtime_error(std::string(what) + ": status " + std::to_string(rc) +
                                 (ctx ? std::string(" (") + swe_last_error(ctx) + ")" : std::string()));
}

// domain + device context (create_domain, src/domain/domain_factory_mod.f90:55-147)
class domain_gpu_t {
  public:
    explicit domain_gpu_t(const swe_cfg &cfg) : cfg_(cfg) { check(swe_ctx_create(&cfg_, &ctx_), nullptr, "swe_ctx_create"); }
    ~domain_gpu_t() { if (ctx_) swe_ctx_destroy(ctx_); }
    domain_gpu_t(const domain_gpu_t &) = delete;
    domain_gpu_t &operator=(const domain_gpu_t &) = delete;
    swe_ctx *ctx() const { return ctx_; }
    const swe_cfg &cfg() const { return cfg_; }

  private:
    swe_cfg cfg_;
    swe_ctx *ctx_ = nullptr;
};

// stvec_swm_t on the device (src/models/shallow_water/stvec/stvec_swm_mod.f90:10-42)
class stvec_swm_gpu_t {
  public:
    explicit stvec_swm_gpu_t(const domain_gpu_t &d) : d_(d) { check(swe_stvec_create(d.ctx(), &v_), d.ctx(), "swe_stvec_create"); }
    ~stvec_swm_gpu_t() { if (v_) swe_stvec_destroy(v_); }
    stvec_swm_gpu_t(const stvec_swm_gpu_t &) = delete;
    stvec_swm_gpu_t &operator=(const stvec_swm_gpu_t &) = delete;
    swe_stvec *handle() const { return v_; }

    // y = s1*v1 + s2*v2 / y = s1*v1 (stvec_flexible_mod.f90:196-250)
    void assign(double s1, const stvec_swm_gpu_t &v1, double s2, const stvec_swm_gpu_t &v2)
    {
        check(swe_stvec_assign(v_, s1, v1.v_, s2, v2.v_), d_.ctx(), "assign");
    }
    void assign(double s1, const stvec_swm_gpu_t &v1) { check(swe_stvec_assign(v_, s1, v1.v_, 0.0, nullptr), d_.ctx(), "assign"); }
    // y = y + s1*v1 + s2*v2 (stvec_flexible_mod.f90:252-306)
    void update(double s1, const stvec_swm_gpu_t &v1, double s2, const stvec_swm_gpu_t &v2)
    {
        check(swe_stvec_update(v_, s1, v1.v_, s2, v2.v_), d_.ctx(), "update");
    }
    void upload(int member, const double *h, const double *u, const double *v)
    {
        check(swe_stvec_upload(v_, member, h, u, v), d_.ctx(), "upload");
    }
    void download(int member, double *h, double *u, double *v) const
    {
        check(swe_stvec_download(v_, member, h, u, v), d_.ctx(), "download");
    }

  private:
    const domain_gpu_t &d_;
    swe_stvec *v_ = nullptr;
};

// operator_swm_lin_t (src/models/shallow_water/operator/operator_swm_lin_mod.f90:66-108)
class operator_swm_lin_gpu_t {
  public:
    explicit operator_swm_lin_gpu_t(const domain_gpu_t &d) : d_(d) {}
    void apply(stvec_swm_gpu_t &vout, const stvec_swm_gpu_t &vin)
    {
        check(swe_operator_apply(d_.ctx(), vout.handle(), vin.handle()), d_.ctx(), "operator apply");
    }
    void integrals(const stvec_swm_gpu_t &s, int member, double &mass, double &energy) const
    {
        check(swe_integrals(d_.ctx(), s.handle(), member, &mass, &energy), d_.ctx(), "integrals");
    }
    const domain_gpu_t &domain() const { return d_; }

  private:
    const domain_gpu_t &d_;
};

// rk4_t (src/time_schemes/rk4_mod.f90:20-42)
class rk4_gpu_t {
  public:
    void step(stvec_swm_gpu_t &v0, operator_swm_lin_gpu_t &op, double dt)
    {
        check(swe_rk4_step(op.domain().ctx(), v0.handle(), dt), op.domain().ctx(), "rk4 step");
    }
    void steps(stvec_swm_gpu_t &v0, operator_swm_lin_gpu_t &op, double dt, int nsteps)
    {
        check(swe_rk4_steps(op.domain().ctx(), v0.handle(), dt, nsteps), op.domain().ctx(), "rk4 steps");
    }
};

// operator_swm_diff_t (src/models/shallow_water/operator/operator_swm_diff_mod.f90:27-49) on the
// Ah staggering: hordiff_vec_xyz_Ah_sbp_<order>_narrow and hordiff_scalar_Ah_sbp_<order>_narrow,
// order 21, 42 (N >= 11) or 63 (N >= 17).
class operator_swm_diff_gpu_t {
  public:
    operator_swm_diff_gpu_t(const domain_gpu_t &d, int order, double uv_coeff, double h_coeff)
        : d_(d), order_(order), uv_(uv_coeff), h_(h_coeff)
    {
    }
    void apply(stvec_swm_gpu_t &vout, const stvec_swm_gpu_t &vin)
    {
        check(swe_diffusion_apply(d_.ctx(), vout.handle(), vin.handle(), order_, uv_, h_), d_.ctx(), "diffusion apply");
    }
    // explicit_Eul1_t%step (src/time_schemes/explicit_Eul1_mod.f90:20-28): v0 += dt apply(v0)
    void euler_step(stvec_swm_gpu_t &v0, double dt)
    {
        check(swe_diffusion_step(d_.ctx(), v0.handle(), dt, order_, uv_, h_), d_.ctx(), "diffusion step");
    }
    // the driver loop (src/models/shallow_water/shallow_water_mod.f90:112-118) on the device:
    // every RK4 step of the domain is followed by euler_step, inside the captured graphs;
    // detach() restores plain RK4 steps
    void attach() { check(swe_set_diffusion(d_.ctx(), order_, uv_, h_), d_.ctx(), "set diffusion"); }
    void detach() { check(swe_set_diffusion(d_.ctx(), 0, 0.0, 0.0), d_.ctx(), "set diffusion"); }

  private:
    const domain_gpu_t &d_;
    int order_;
    double uv_, h_;
};

// Several domains' RK4 steps as one grid per kernel (swe_group_*: up to 8 linear Ch
// contexts of one precision and split kernel configuration, any cube sizes); no
// reference counterpart, the reference advances one state per timescheme%step.
class group_gpu_t {
  public:
    explicit group_gpu_t(const std::vector<const domain_gpu_t *> &doms)
    {
        std::vector<swe_ctx *> c;
        for (const domain_gpu_t *d : doms) c.push_back(d->ctx());
        check(swe_group_create(c.data(), (int)c.size(), &g_), c.empty() ? nullptr : c[0], "swe_group_create");
    }
    ~group_gpu_t() { if (g_) swe_group_destroy(g_); }
    group_gpu_t(const group_gpu_t &) = delete;
    group_gpu_t &operator=(const group_gpu_t &) = delete;
    // nsteps RK4 steps of states[k] with the per-member time steps dts[k]
    void steps_members(const std::vector<stvec_swm_gpu_t *> &states, const std::vector<const double *> &dts, int nsteps)
    {
        std::vector<swe_stvec *> v;
        for (stvec_swm_gpu_t *s : states) v.push_back(s->handle());
        const int rc = swe_group_rk4_steps_members(g_, v.data(), dts.data(), nsteps);
        if (rc != SWE_OK)
            throw std::runtime_error(std::string("group steps: status ") + std::to_string(rc) + " (" +
                                     swe_group_last_error(g_) + ")");
    }

  private:
    swe_group *g_ = nullptr;
};

}  // namespace chswe_host
