// Oracle C entry points -- TEST INFRASTRUCTURE ONLY (loaded by tests/ and bench.py's CPU
// baseline through ctypes).  Wraps the kernel-form restatement (kernel_form.hpp) in the
// same argument conventions as include/hp2d.h so a test can drive the CUDA library and
// the oracle with identical calls.
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "kernel_form.hpp"

using hp2d_oracle::Model;

struct oracle_model {
    int precision;
    std::unique_ptr<Model<float>> f;
    std::unique_ptr<Model<double>> d;
};

template <typename F> static int dispatch(oracle_model* m, F&& fn) {
    if (!m) return HP2D_INVALID_ARG;
    if (m->precision == HP2D_FP32) return fn(*m->f);
    return fn(*m->d);
}

extern "C" {

oracle_model* oracle_create(const hp2d_grid* g, const hp2d_params* p) {
    auto* m = new oracle_model();
    m->precision = g->precision;
    if (g->precision == HP2D_FP32) m->f.reset(new Model<float>(*g, *p));
    else m->d.reset(new Model<double>(*g, *p));
    return m;
}

void oracle_destroy(oracle_model* m) { delete m; }

int oracle_upload_static(oracle_model* m, const double* z, const double* n, const int32_t* rows,
                         const int32_t* cols, int32_t nout, const double* slopes) {
    return dispatch(m, [&](auto& M) { M.upload_static(z, n, rows, cols, nout, slopes); return 0; });
}

int oracle_set_soil(oracle_model* m, const uint8_t* cls, int32_t ncls, const double* ksat,
                    const double* psi, const double* dtheta, const double* Lu, const double* kout,
                    const double* Tr, const double* minsm) {
    return dispatch(m, [&](auto& M) {
        M.set_soil(cls, ncls, ksat, psi, dtheta, Lu, kout, Tr, minsm);
        return 0;
    });
}

int oracle_set_state(oracle_model* m, const double* d, const double* outflow, const double* I) {
    return dispatch(m, [&](auto& M) { M.set_state(d, outflow, I); return 0; });
}

int oracle_set_depth(oracle_model* m, const double* d) {
    return dispatch(m, [&](auto& M) { M.set_depth(d); return 0; });
}

int oracle_set_clock(oracle_model* m, double t, double time_step, int64_t k) {
    return dispatch(m, [&](auto& M) {
        M.set_clock(t, time_step, k);
        return 0;
    });
}

int oracle_set_inflow(oracle_model* m, int32_t ng, int32_t nt, const double* t0, const double* rate, int32_t nc,
                      const int32_t* rows, const int32_t* cols, const int32_t* gauge, const double* z) {
    return dispatch(m, [&](auto& M) {
        M.set_inflow(ng, nt, t0, rate, nc, rows, cols, gauge, z);
        return 0;
    });
}

int oracle_set_stage(oracle_model* m, int32_t ng, int32_t nt, const double* t0, const double* d, int32_t nc,
                     const int32_t* rows, const int32_t* cols, const int32_t* gauge) {
    return dispatch(m, [&](auto& M) { M.set_stage(ng, nt, t0, d, nc, rows, cols, gauge); return 0; });
}

int oracle_set_reservoirs(oracle_model* m, int32_t n, const int32_t* rr, const int32_t* rc, const double* k1,
                          const double* h1, const double* k2, const int32_t* d1r, const int32_t* d1c, const double* k3,
                          const double* h2, const double* k4, const int32_t* d2r, const int32_t* d2c) {
    return dispatch(m, [&](auto& M) { M.set_reservoirs(n, rr, rc, k1, h1, k2, d1r, d1c, k3, h2, k4, d2r, d2c); return 0; });
}

int oracle_set_hazard_tracking(oracle_model* m, int32_t on) {
    return dispatch(m, [&](auto& M) { M.set_hazard_tracking(on != 0); return 0; });
}

int oracle_set_map_records(oracle_model* m, int32_t n, const double* times) {
    return dispatch(m, [&](auto& M) { M.set_map_records(n, times); return 0; });
}

int64_t oracle_map_records(oracle_model* m) {
    return dispatch(m, [&](auto& M) { return int64_t(M.rec_maps.size()); });
}

// record `index`: depth [mm] as the library converts it (state precision -> double x 1000)
int oracle_download_map_record(oracle_model* m, int64_t index, double* depth_mm, double* t_min) {
    return dispatch(m, [&](auto& M) {
        if (index < 0 || size_t(index) >= M.rec_maps.size()) return 1;
        const auto& v = M.rec_maps[size_t(index)];
        for (size_t k = 0; k < v.size(); ++k) depth_mm[k] = double(v[k]) * 1000.0;
        *t_min = M.rec_t[size_t(index)];
        return 0;
    });
}

int oracle_set_rain_clock(oracle_model* m, double a, double b, double t_previous) {
    return dispatch(m, [&](auto& M) {
        M.rain_a = a;
        M.rain_b = b;
        M.t_prev = t_previous;
        return 0;
    });
}

int oracle_set_rain_uniform(oracle_model* m, int32_t n, const double* t0, const double* rate) {
    return dispatch(m, [&](auto& M) {
        M.rain_t.assign(t0, t0 + n);
        M.rain_r.assign(rate, rate + n);
        M.n_maps = 0;
        return 0;
    });
}

int oracle_set_rain_maps(oracle_model* m, int32_t nm, int32_t my, int32_t mx, const float* rate,
                         double map_dt) {
    return dispatch(m, [&](auto& M) {
        M.n_maps = nm; M.my = my; M.mx = mx; M.map_dt = map_dt;
        M.map_t.clear();
        M.maps.assign(rate, rate + size_t(nm) * my * mx);
        return 0;
    });
}

// end-stamped input maps: map q over [t_end[q-1], t_end[q]), the first from t_end[0] - dt_force
// (localAverageInputRainMapOverStep, update_spatial_BC.m:1287-1359)
int oracle_set_rain_maps_end_stamped(oracle_model* m, int32_t nm, int32_t my, int32_t mx, const float* rate,
                                     const double* t_end, double dt_force) {
    return dispatch(m, [&](auto& M) {
        M.n_maps = nm; M.my = my; M.mx = mx; M.map_dt = 0.0;
        M.map_t.assign(size_t(nm) + 1, 0.0);
        M.map_t[0] = t_end[0] - dt_force;
        for (int q = 0; q < nm; ++q) M.map_t[size_t(q) + 1] = t_end[q];
        M.maps.assign(rate, rate + size_t(nm) * my * mx);
        return 0;
    });
}

int oracle_hydrology_step(oracle_model* m, double time_step) {
    return dispatch(m, [&](auto& M) { M.hydrology(time_step * 60.0); return 0; });
}

int oracle_li_step(oracle_model* m, double time_step) {
    return dispatch(m, [&](auto& M) { M.li(time_step * 60.0, time_step); return 0; });
}

int oracle_cfl_dt(oracle_model* m, double time_step_applied, double* ts_out, double* vmax) {
    return dispatch(m, [&](auto& M) {
        double tcr = M.cfl(time_step_applied * 60.0, vmax);
        *ts_out = tcr / 60.0;
        return 0;
    });
}

int oracle_track_maxima(oracle_model* m, double t_end) {
    return dispatch(m, [&](auto& M) { M.track(t_end * 60.0); return 0; });
}

}  // extern "C"

// nsteps accepted steps (as hp2d_fused_steps): a rejected attempt is retried in place; the
// call returns HP2D_NUMERICAL when one step's retries run out or the state holds a NaN depth
// in a cell of finite elevation, HP2D_DT_FLOOR after a step that hit min_time_step with the
// dt-floor stop on
template <typename M_> static int accepted_steps(M_& M, int64_t nsteps, int64_t* done) {
    if (M.bad_domain()) return int(HP2D_NUMERICAL);
    M.n_bad0 = M.count_bad(false);
    const int64_t k0 = M.k;
    int st = 0;
    while (M.k - k0 < nsteps && !M.finished()) {
        const int r = M.step();
        if (r == M_::kFailed) { st = int(HP2D_NUMERICAL); break; }
        if (r == M_::kDtFloor) { st = int(HP2D_DT_FLOOR); break; }
    }
    if (done) *done = M.k - k0;
    return st;
}

extern "C" {

int oracle_steps(oracle_model* m, int32_t nsteps) {
    return dispatch(m, [&](auto& M) { return accepted_steps(M, nsteps, nullptr); });
}

int oracle_run(oracle_model* m, int64_t max_steps, int64_t* done) {
    return dispatch(m, [&](auto& M) {
        return accepted_steps(M, max_steps > 0 ? max_steps : (int64_t(1) << 40), done);
    });
}

int oracle_set_retry_policy(oracle_model* m, int32_t max_retries, double factor_reduction, int32_t dt_floor_is_error) {
    return dispatch(m, [&](auto& M) {
        M.max_retries = max_retries;
        M.factor_reduction = factor_reduction;
        M.dt_floor_stop = dt_floor_is_error;
        return 0;
    });
}

int oracle_set_refresh_every(oracle_model* m, int32_t k) {
    return dispatch(m, [&](auto& M) {
        M.refresh_every = k;
        return 0;
    });
}

int oracle_inject_step_fault(oracle_model* m, int64_t k, int32_t attempts) {
    return dispatch(m, [&](auto& M) {
        M.fault_k = k;
        M.fault_n = attempts;
        return 0;
    });
}

// Raw state in the internal units and precision (for bit-exact comparison).
//   0 h [m], 1 qx [m^2/s], 2 qy, 3 I [m], 4 T [s], 5 dmax [m], 6 arrival [s],
//   7 Hf_x [m], 8 Hf_y [m], 9 Hf3 per outlet, 10 outlet rate per outlet [m/s],
//   11 velocity maximum [m/s], 12 hazard maximum [m^2/s]
int oracle_download_native(oracle_model* m, int32_t field, void* out, size_t bytes) {
    return dispatch(m, [&](auto& M) {
        using R = typename std::remove_reference<decltype(M.h[0])>::type;
        const std::vector<R>* src = nullptr;
        switch (field) {
            case 0: src = &M.h; break;
            case 1: src = &M.qx; break;
            case 2: src = &M.qy; break;
            case 3: src = &M.I; break;
            case 4: src = &M.T; break;
            case 5: src = &M.dmax; break;
            case 6: src = &M.arrival; break;
            case 7: src = &M.hfx; break;
            case 8: src = &M.hfy; break;
            case 9: src = &M.hf3; break;
            case 10: src = &M.qo; break;
            case 11: src = &M.vmaxm; break;
            case 12: src = &M.hzmaxm; break;
            default: return int(HP2D_INVALID_ARG);
        }
        if (bytes != src->size() * sizeof(R)) return int(HP2D_INVALID_ARG);
        std::memcpy(out, src->data(), bytes);
        return 0;
    });
}

// x^(7/3), x^(5/3) of the deterministic Newton iteration, for accuracy tests
void oracle_pow_check(int32_t precision, int32_t n, const double* x, double* p73, double* p53) {
    for (int i = 0; i < n; ++i) {
        if (precision == 0) {
            p73[i] = double(hp2d_oracle::pow73<float>(float(x[i])));
            p53[i] = double(hp2d_oracle::pow53<float>(float(x[i])));
        } else {
            p73[i] = hp2d_oracle::pow73<double>(x[i]);
            p53[i] = hp2d_oracle::pow53<double>(x[i]);
        }
    }
}

void oracle_qdiv_check(int32_t n, const float* a, const float* b, float* q) {
    for (int i = 0; i < n; ++i) q[i] = hp2d_oracle::qdiv(a[i], b[i]);
}

int oracle_get_diag(oracle_model* m, hp2d_diag* o) {
    return dispatch(m, [&](auto& M) {
        o->t = M.t_min;
        o->time_step = M.time_step;
        o->k = M.k;
        o->max_velocity = M.vmax_last;
        o->rain_volume = M.rain_vol;
        o->infiltration_volume = M.inf_vol;
        o->outlet_volume = M.out_vol;
        o->neg_depth_warnings = M.neg_warn;
        o->unstable_steps = M.unstable;
        o->status_bits = 0;
        o->rain_t0 = M.rain_a;
        o->rain_t1 = M.rain_b;
        o->t_previous = M.t_prev;
        o->inflow_volume = M.inflow_vol;
        o->stage_volume = M.stage_vol;
        o->structure_volume = M.struct_vol;
        o->skipped_cells = 0;
        o->skipped_read_cells = 0;
        o->retries = M.retries;
        o->catch_index = M.catch_index;
        o->steps_per_block = M.refresh_every;
        o->max_time_step = M.max_dt();
        return 0;
    });
}

}  // extern "C"
