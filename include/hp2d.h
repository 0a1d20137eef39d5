/*
 * hp2d.h -- C ABI of the B200 surface-flow step for HydroPol2D.
 *
 * One context (hp2d_ctx) holds one grid resident in GPU memory.  The entry points
 * replace, one for one, the MATLAB functions and scripts that HydroPol2D_Main_While
 * calls on its surface-flow path:
 *
 *   hp2d_hydrology_step  rain (interception_module.m:68-71, Snow_Module.m:99), the
 *                        Infiltration_Module script (Green-Ampt form, see below) and
 *                        the depth clamp of Hydrological_Model.m:45-55
 *   hp2d_li_step         Local_Inertial_Model_D4.m:1-5 (+ Inertial_Solver.m:1, scheme 1)
 *   hp2d_cfl_dt          refreshing_timestep.m:17-359 (inertial, D4)
 *   hp2d_track_maxima    save_output_maps.m:588-600 (running maximum depth) + arrival time
 *   hp2d_fused_steps     all of the above, one fused kernel per accepted step, in the
 *                        order of HydroPol2D_Main_While.m:403-782
 *
 * Conventions at this boundary (the MATLAB units): depths in mm, face fluxes in mm/h
 * referenced to the cell area, time steps in minutes, the clock in minutes, elevations
 * in m.  Arrays are row-major with x (MATLAB's column index) fastest: element (i, j) of a
 * MATLAB ny-by-nx array is at i*nx + j.  A MEX gateway transposes column-major data on
 * the way in and out.  Inside, the state is SI (m, m^2/s, s).
 *
 * Every call returns an hp2d_status; on failure hp2d_last_error() gives a message.
 * Host pointers are borrowed for the duration of the call only.  Calls on one context
 * are synchronous with respect to the host and must come from one host thread at a time.
 */
#ifndef HP2D_H
#define HP2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hp2d_status {
    HP2D_OK = 0,
    HP2D_INVALID_ARG = 1,
    HP2D_UNSUPPORTED_FLAG = 2,   /* flag_subgrid/flag_D8=1, scheme 2/3 ... */
    HP2D_CUDA_ERROR = 3,
    HP2D_NUMERICAL = 4,          /* a step kept failing (non-finite or negative depth), or the state
                                    holds a NaN depth in a cell of finite elevation */
    HP2D_DT_FLOOR = 5,           /* dt hit min_time_step (refreshing_timestep.m:357-359), with
                                    hp2d_set_retry_policy's dt_floor_is_error = 1 */
    HP2D_TIMEOUT = 6,            /* a row copy into shared memory did not land within the wait
                                    limit (hp2d_set_wait_limit); that step was rejected */
    HP2D_NO_DEVICE = 7,
    HP2D_NOT_READY = 8           /* static data or state not uploaded yet */
} hp2d_status;

typedef enum hp2d_precision { HP2D_FP32 = 0, HP2D_FP64 = 1 } hp2d_precision;

typedef struct hp2d_grid {
    int32_t ny;            /* rows    (MATLAB size(z,1)) */
    int32_t nx;            /* columns (MATLAB size(z,2)) */
    double resolution;     /* Wshed_Properties.Resolution [m]; cell_area = resolution^2 */
    int32_t precision;     /* hp2d_precision of the state and of the per-cell arithmetic */
} hp2d_grid;

/* Flags and controls the path reads (Config/input_data_bypass_script.m:160-170, :330-380,
 * input_data_script.m:92-154).  Unsupported values are rejected, never ignored. */
typedef struct hp2d_params {
    int32_t flag_numerical_scheme;      /* 1 (Bates); 2 and 3 -> HP2D_UNSUPPORTED_FLAG */
    int32_t flag_critical;              /* 0/1: critical-velocity clip (LIM_D4.m:272-275) */
    int32_t flag_subgrid;               /* must be 0 */
    int32_t flag_D8;                    /* must be 0 */
    int32_t flag_reservoir;             /* 0, or 1 with hp2d_set_reservoirs */
    int32_t flag_infiltration;          /* 0 off, 1 Green-Ampt (hp2d_set_soil), 2 van Genuchten (hp2d_set_soil_vg) */
    int32_t flag_timestep;              /* 1: dt = min(dt_adv, dt_wave); 0: dt_wave */
    int32_t flag_adaptive_timestepping; /* 1: wave celerity only; 0: celerity + speed */
    int32_t outlet_type;                /* 1 normal-depth slope, 2 critical */
    double slope_outlet;                /* [m/m], outlet_type 1 */
    double min_time_step;               /* running_control.min_time_step [s] */
    double max_time_step;               /* running_control.max_time_step [s] */
    double time_step_increments;        /* [s] */
    double time_step_change;            /* [s] refresh gate of HydroPol2D_Main_While.m:691-695 */
    double routing_time;                /* [min] end of the simulation */
    double alfa_min;                    /* Courant_Parameters.alfa_min */
    double alfa_max;                    /* Courant_Parameters.alfa_max */
    double depth_tolerance;             /* CA_States.depth_tolerance [mm] */
    double arrival_threshold;           /* depth defining the arrival time [mm] */
} hp2d_params;

/* Fields for hp2d_download.  Units are the MATLAB ones. */
typedef enum hp2d_field {
    HP2D_FIELD_DEPTH = 0,        /* depths.d_t [mm] */
    HP2D_FIELD_QOUT_RIGHT = 1,   /* flow_rate.qout_right_t = outflow_bates(:,:,1) [mm/h] */
    HP2D_FIELD_QOUT_UP = 2,      /* flow_rate.qout_up_t    = outflow_bates(:,:,2) [mm/h] */
    HP2D_FIELD_QOUT_LEFT = 3,    /* flow_rate.qout_left_t  [mm/h] (LIM_D4.m:347) */
    HP2D_FIELD_QOUT_DOWN = 4,    /* flow_rate.qout_down_t  [mm/h] (LIM_D4.m:350) */
    HP2D_FIELD_OUTLET_FLOW = 5,  /* outlet_states.outlet_flow = outflow_bates(:,:,3) [mm/h] */
    HP2D_FIELD_HF_X = 6,         /* Hf(:,:,1) [m] of the last li step */
    HP2D_FIELD_HF_Y = 7,         /* Hf(:,:,2) [m] */
    HP2D_FIELD_HF_OUTLET = 8,    /* Hf(:,:,3) [m] */
    HP2D_FIELD_DMAX = 9,         /* depths.dmax_final [mm] */
    HP2D_FIELD_ARRIVAL = 10,     /* first time depth >= arrival_threshold [min]; +Inf never */
    HP2D_FIELD_SOIL_STORAGE = 11,/* Soil_Properties.I_t [mm] */
    HP2D_FIELD_I_TOT_END_CELL = 12,/* CA_States.I_tot_end_cell [m^3] (LIM_D4.m:512-514) */
    HP2D_FIELD_VMAX = 13,        /* velocities.vmax_final [m/s] (hp2d_set_hazard_tracking) */
    HP2D_FIELD_HAZARD_MAX = 14   /* velocities.hazardmax_final, depth x velocity [m^2/s] */
} hp2d_field;

typedef struct hp2d_diag {
    double t;                     /* clock [min] */
    double time_step;             /* step the next call applies [min] */
    int64_t k;                    /* step counter (1-based, as the reference) */
    double max_velocity;          /* velocities.max_velocity of the last refresh [m/s] */
    double rain_volume;           /* cumulative [m^3] */
    double infiltration_volume;   /* cumulative [m^3] */
    double outlet_volume;         /* cumulative [m^3] */
    int64_t neg_depth_warnings;   /* Hydrological_Model.m:45-47 events */
    int64_t unstable_steps;       /* refreshing_timestep.m:357-359 events */
    int64_t status_bits;          /* bit 0: a step was rejected for its depths; bit 1: a row copy
                                     timed out; bit 2: the refreshed dt hit min_time_step */
    double rain_t0, rain_t1;      /* clock interval whose rain the next step applies [min] */
    double t_previous;            /* the loop's t_previous [min] */
    double inflow_volume;         /* cumulative inflow-hydrograph volume [m^3] */
    double stage_volume;          /* cumulative volume the stage overwrites added [m^3] */
    double structure_volume;      /* cumulative volume the control structures added [m^3] */
    int64_t skipped_cells;        /* cumulative cell records the fused step found already
                                     written (dry rows) and did not store again */
    int64_t skipped_read_cells;   /* of those, cells of whole dry row blocks whose records
                                     were not read either */
    int64_t retries;              /* rejected step attempts retried so far */
    int32_t catch_index;          /* the reference's catch_index (1 + failures so far) */
    int32_t steps_per_block;      /* temporal blocking in use (1: off; hp2d_set_temporal_blocking) */
    double max_time_step;         /* running_control.max_time_step [s], lowered by retries */
} hp2d_diag;

typedef struct hp2d_ctx hp2d_ctx;

/* ---- lifetime --------------------------------------------------------------------- */
/* Creates a context on CUDA device `device`.  Replaces the gpuArray set-up of
 * HydroPol2D_preprocessing.m:2754-2771 for the arrays of this path. */
hp2d_status hp2d_create(const hp2d_grid* grid, const hp2d_params* params, int32_t device,
                        hp2d_ctx** out);
hp2d_status hp2d_destroy(hp2d_ctx* ctx);
const char* hp2d_last_error(const hp2d_ctx* ctx);
/* Library-wide message of the last failed hp2d_create (no context exists then). */
const char* hp2d_create_error(void);

/* ---- inputs ----------------------------------------------------------------------- */
/* Elevation_Properties.elevation_cell [m] (NaN = idx_nan cell, a wall),
 * LULC_Properties.roughness (roughness_squared = roughness.^2, Main_While.m:188),
 * Wshed_Properties.row_outlet/col_outlet (0-based) and, optionally, one slope per outlet
 * cell (slope_outlet given as a map); NULL uses params.slope_outlet. */
hp2d_status hp2d_upload_static(hp2d_ctx* ctx, const double* z, const double* roughness,
                               const int32_t* outlet_rows, const int32_t* outlet_cols,
                               int32_t n_outlets, const double* slope_outlet_per_outlet);

/* Green-Ampt soil classes: class map (255 = no soil: impervious, no infiltration) and
 * per-class tables.  ksat [mm/h], psi [mm], dtheta = teta_sat - teta_i [-], Lu [m],
 * k_out [mm/h], Tr [h] and min_soil_moisture [mm] as HydroPol2D_preprocessing.m:2250-2253
 * and :2387-2388 define them. */
hp2d_status hp2d_set_soil(hp2d_ctx* ctx, const uint8_t* soil_class, int32_t n_classes,
                          const double* ksat, const double* psi, const double* dtheta,
                          const double* Lu, const double* k_out, const double* Tr,
                          const double* min_soil_moisture);

/* van Genuchten-Mualem soil (the single-layer branch of the current Infiltration_Module.m,
 * :143-473; flag_infiltration = 2): class map (255 = no soil) and per-class theta_r,
 * theta_sat [-], n_vg [-] (> 1), alpha_vg [1/m], ksat [mm/h]; per cell Soil_Depth [m] and
 * the groundwater head BC_States.h_t [m] (NULL = water table at the soil bottom); the
 * scalars Soil_Properties.l_vg, Ltop [m], dh_max [m] and Ksurf_weight (reference defaults
 * 0.5, 0.05, 1.0, 0.5).  Call after hp2d_upload_static (the water-table depth uses the DEM).
 * Soil storage I_t [mm] comes with hp2d_set_state. */
hp2d_status hp2d_set_soil_vg(hp2d_ctx* ctx, const uint8_t* soil_class, int32_t n_classes,
                             const double* theta_r, const double* theta_sat, const double* n_vg,
                             const double* alpha_vg, const double* ksat, const double* soil_depth,
                             const double* gw_head, double l_vg, double Ltop, double dh_max,
                             double ksurf_weight);

/* State: depths.d_t [mm]; outflow_bates pages 1-2 [mm/h] (two ny*nx blocks, right then
 * up; NULL = zeros); Soil_Properties.I_t [mm] (NULL = keep).  Resets dmax and arrival. */
hp2d_status hp2d_set_state(hp2d_ctx* ctx, const double* d, const double* outflow,
                           const double* soil_storage);

/* Clock [min], the step the next call applies [min] and the step counter k (1-based).
 * The rain interval follows it: k = 1 starts a run (interval [0, t], t_previous 0); k one
 * above the current counter is the loop's advance (HydroPol2D_Main_While.m:721-779: the
 * interval becomes [t_previous, previous clock], t_previous becomes time_step after the
 * first step and the previous clock after that); any other k re-seeds the interval as if
 * the last two steps had taken time_step. */
hp2d_status hp2d_set_clock(hp2d_ctx* ctx, double t, double time_step, int64_t k);

/* The rain interval [rain_t0, rain_t1] [min] whose rain the next step applies and the loop's
 * t_previous [min] (the update_spatial_BC state; hp2d_get_diag reports them), for an exact
 * restart. */
hp2d_status hp2d_set_rain_clock(hp2d_ctx* ctx, double rain_t0, double rain_t1, double t_previous);

/* Rain forcing.  A step applies the rain of a clock interval, as update_spatial_BC.m does
 * at the end of the step before it: the exact integral of the piecewise-constant rate
 * over the interval (:435-470, :1131-1184; maps :536-558, :1287-1359), / 60 -> mm.
 * Uniform: rates [mm/h] holding from t_start[q] [min] up to t_start[q+1], the last one for
 * ever (an end-stamped series converts by prepending its first start and appending a
 * zero rate).  Maps: n_maps coarse fields (my x mx, row-major) [mm/h], map m holding over
 * [m*map_dt, (m+1)*map_dt) [min] and nothing after the last one, bilinearly interpolated
 * to the grid; map_dt*60 must be at least params.max_time_step [s] (a step's interval then
 * overlaps at most two maps). */
hp2d_status hp2d_set_rain_uniform(hp2d_ctx* ctx, int32_t n, const double* t_start,
                                  const double* rate);
hp2d_status hp2d_set_rain_maps(hp2d_ctx* ctx, int32_t n_maps, int32_t my, int32_t mx,
                               const float* rate, double map_dt);
/* Input rain maps (flags.flag_input_rainfall_map = 1; update_spatial_BC.m:497-517 with
 * localAverageInputRainMapOverStep :1287-1359): end-stamped rate maps [mm/h], map m holding
 * over [t_end[m-1], t_end[m]) [min] and the first one from t_end[0] - dt_force (the reference's
 * Input_Rainfall.time and dt_force, by default t_end[1] - t_end[0]), nothing after the last.
 * The maps are given already aligned to the grid (my x mx, bilinearly sampled as above; at
 * my = ny, mx = nx each cell takes its own value): hydropol2d_b200.raster_rain reads GeoTIFF
 * rasters and aligns them as raster_cutter.m does.  Each non-empty interval must be at least
 * params.max_time_step long. */
hp2d_status hp2d_set_rain_maps_end_stamped(hp2d_ctx* ctx, int32_t n_maps, int32_t my, int32_t mx,
                                           const float* rate, const double* t_end, double dt_force);

/* Rain from gauges (flags.flag_spatial_rainfall = 1; update_spatial_BC.m:494-517 with
 * Rainfall_Interpolator.m / idw_function.m): n_gauges at eastings/northings x_gauge, y_gauge
 * [m] record rates [mm/h] (row-major [n_times][n_gauges], NaN = no record) over intervals of
 * record_dt minutes, interval m over [m, m+1) * record_dt.  The library interpolates one map
 * per interval by inverse-distance weighting (power 2, Euclidean distance, no radius) at the
 * cell centres (x_ul + res (j+1), y_ul - res (i+1)) (HydroPol2D_preprocessing.m:2420-2421) and
 * uses them as rain maps (hp2d_set_rain_maps semantics; record_dt*60 >= max_time_step). */
hp2d_status hp2d_set_rain_gauges(hp2d_ctx* ctx, int32_t n_gauges, const double* x_gauge, const double* y_gauge,
                                 int32_t n_times, double record_dt, const double* rates, double x_ul, double y_ul);

/* Inflow hydrographs (flags.flag_inflow = 1; update_spatial_BC.m:359-395): n_gauges rate
 * series [mm/h] (rates row-major [n_times][n_gauges]) on the start-stamped table t_start
 * [min] (rate q holds from t_start[q] up to t_start[q+1], the last for ever), and the
 * n_cells (rows, cols, gauge) entries of Wshed_Properties.inflow_cells(:,:,gauge) (a cell may
 * belong to several gauges).  Each step adds to a cell, after the infiltration
 * (Hydrological_Model.m:27-28), the integral of its gauges' rates over the step's rain
 * interval / 60 mm (BC_States.inflow).  Call after hp2d_upload_static (which removes the
 * inflow); an outlet cell cannot be an inflow cell; n_gauges = 0 removes the inflow. */
hp2d_status hp2d_set_inflow(hp2d_ctx* ctx, int32_t n_gauges, int32_t n_times, const double* t_start,
                            const double* rates, int32_t n_cells, const int32_t* rows, const int32_t* cols,
                            const int32_t* gauge);

/* Map records (save_output_maps.m:25-27, :160-166): after a step whose t_save = t + the new
 * step (HydroPol2D_Main_While.m:740) passes one or more of the record times
 * (running_control.time_records [min], increasing), the depth d_t after that step is kept on
 * the device with the step's clock t; n_slots maps are held, the oldest overwritten first.
 * The first-step map the reference writes before any record event is overwritten by the first
 * event there and is not kept here.  n_times = 0 switches the records off. */
hp2d_status hp2d_set_map_records(hp2d_ctx* ctx, int32_t n_times, const double* time_records, int32_t n_slots);
/* hp2d_set_map_records with the n_slots maps kept in page-locked host memory mapped into the
 * device's address space (no counterpart in the reference; save_output_maps.m:565-580 moves the
 * maps to the host in chunks): the step that takes a record writes the map across the host link
 * itself, overlapped with the rest of its work, so no copy runs at read-back time and nothing of
 * the record ring occupies GPU memory.  Read with hp2d_download_map_record as usual. */
hp2d_status hp2d_set_map_records_host(hp2d_ctx* ctx, int32_t n_times, const double* time_records, int32_t n_slots);
/* Records taken so far. */
hp2d_status hp2d_map_records(hp2d_ctx* ctx, int64_t* count);
/* Record `index` (0-based, one of the last n_slots taken): depth [mm] (ny*nx) and clock [min]. */
hp2d_status hp2d_download_map_record(hp2d_ctx* ctx, int64_t index, double* depth_mm, double* t_min);

/* Stage hydrographs (flags.flag_stage_hydrograph = 1; update_spatial_BC.m:316-357): n_gauges
 * water-depth series [m] (row-major [n_times][n_gauges]) on the start-stamped table t_start
 * [min] (the record in force is the last starting at or before the clock, else the first),
 * and the n_cells (rows, cols, gauge) of Wshed_Properties.stage_mask(:,:,gauge).  After each
 * fused step (after its timestep refresh, before the maxima) a stage cell's depth becomes its
 * gauge's depth at the step's clock; a cell in several masks takes the highest gauge.  Call
 * after hp2d_upload_static; outlet and NaN-elevation cells cannot be stage cells; the unfused
 * entry points leave the stage to the caller (it is update_spatial_BC's). */
hp2d_status hp2d_set_stage(hp2d_ctx* ctx, int32_t n_gauges, int32_t n_times, const double* t_start,
                           const double* depth_m, int32_t n_cells, const int32_t* rows, const int32_t* cols,
                           const int32_t* gauge);

/* Reservoir / control structures (flag_reservoir = 1): the reservoir_x, reservoir_y, k1, h1,
 * k2, k3, h2, k4, yds1, xds1, yds2, xds2 arguments of Local_Inertial_Model_D4
 * (Local_Inertial_Model_D4.m:2, :318-344; Reservoir_Data of HydroPol2D_preprocessing.m:820-826),
 * 0-based cells, ds1_row = -1 / ds2_row = -1 for the reference's NaN.  Each step, structure i
 * takes the depth of its reservoir cell entering the fluxes and moves
 * dh = min(k1 max(h-h1,0)^k2 / A x 3.6e6, 1000 max(h-h1,0)/dt_h) dt_h [mm] to ds1 (and likewise
 * through k3, h2, k4 to ds2), in structure order, with the reference's bookkeeping: the
 * reservoir cell's volume term GAINS the transfer and the first transfer is added to ds1 a
 * second time when a second structure exists.  The transfers enter each cell after the fluxes
 * (both hp2d_li_step and the fused step); hp2d_get_diag reports the volume they add.  After
 * hp2d_upload_static; outlet and NaN-elevation cells cannot take part; ds2 needs ds1;
 * n = 0 removes them. */
hp2d_status hp2d_set_reservoirs(hp2d_ctx* ctx, int32_t n, const int32_t* res_row, const int32_t* res_col,
                                const double* k1, const double* h1, const double* k2, const int32_t* ds1_row,
                                const int32_t* ds1_col, const double* k3, const double* h2, const double* k4,
                                const int32_t* ds2_row, const int32_t* ds2_col);

/* Velocity and hazard maxima of save_output_maps.m:588-604: each fused step keeps, per cell,
 * the running maximum of the velocity raster max(|vel_left|, |vel_right|, |vel_up|,
 * |vel_down|) of refreshing_timestep.m:109-111 and of snisb_velocity_hazard_snapshot's depth x
 * velocity (0 below 0.01 m, NaN where the depth is NaN).  on = 1 starts both at zero, 0 stops
 * them; read with HP2D_FIELD_VMAX / HP2D_FIELD_HAZARD_MAX.  The reference keeps the raster of
 * its last velocity refresh, so the fused step's maps equal it when every step refreshes:
 * on = 1 needs time_step_change <= min_time_step / 2.  Fused path only. */
hp2d_status hp2d_set_hazard_tracking(hp2d_ctx* ctx, int32_t on);

/* The fused step skips what it can prove unchanged (on by default): a deep-dry row whose output
 * buffer already holds it is not stored again, and a block of rows whose inputs and outputs are
 * all dry (no rain or infiltration that step) is neither read nor written.  Results are the
 * same bit for bit either way; on = 0 runs every row densely (no reference counterpart). */
hp2d_status hp2d_set_dry_skip(hp2d_ctx* ctx, int32_t on);

/* ---- unfused drop-in entry points (one reference function each) ------------------ */
/* Hydrological_Model for this path: adds delta_p_agg (the rain of the current rain
 * interval, see hp2d_set_rain_uniform),
 * runs the Infiltration_Module (Green-Ampt when flag_infiltration=1, van Genuchten when 2)
 * and the clamp; the
 * resident depth becomes d_tot. */
hp2d_status hp2d_hydrology_step(hp2d_ctx* ctx, double time_step);
/* Local_Inertial_Model_D4 on the resident d_tot and outflow_prev with time_step [min];
 * the resident depth becomes d_t and the resident fluxes outflow_bates. */
hp2d_status hp2d_li_step(hp2d_ctx* ctx, double time_step);
/* refreshing_timestep's refresh branch on the last li step's Hf and fluxes: returns the
 * new time_step [min] (= time_calculation_routing/60) and the maximum velocity [m/s]. */
hp2d_status hp2d_cfl_dt(hp2d_ctx* ctx, double* time_step, double* max_velocity);
/* save_output_maps' running maximum depth, and the arrival time t_end [min] for cells
 * whose depth first reaches params.arrival_threshold. */
hp2d_status hp2d_track_maxima(hp2d_ctx* ctx, double t_end);

/* ---- fused path ------------------------------------------------------------------ */
/* Runs `nsteps` accepted steps of HydroPol2D_Main_While.m:403-782 (hydrology, routing,
 * timestep refresh, maxima, clock), one fused kernel per step, launched from a CUDA
 * graph.  Steps after the clock passes routing_time are no-ops. */
hp2d_status hp2d_fused_steps(hp2d_ctx* ctx, int32_t nsteps);
/* hp2d_fused_steps bracketed by CUDA events on the context's stream; *elapsed_ms is the
 * device time of the nsteps launches (for benchmarking). */
hp2d_status hp2d_fused_steps_timed(hp2d_ctx* ctx, int32_t nsteps, float* elapsed_ms);
/* Launch shape of the fused kernel: rows each warp streams through (>= 4; FP32 default 40,
 * FP64 64).  Results do not depend on it; hp2d_autotune times the candidates per grid. */
hp2d_status hp2d_set_tuning(hp2d_ctx* ctx, int32_t rows_per_warp);
/* Layout of the fused kernel: cells each lane streams side by side (1: 32-column strips
 * with 28 output columns; 2: 64-column strips with 60).  Results do not depend on it;
 * hp2d_autotune picks it with the rows per warp. */
hp2d_status hp2d_set_layout(hp2d_ctx* ctx, int32_t cells_per_lane);
/* Autotuner (no counterpart in the reference): times `trial_steps` fused steps from the
 * current state for each launch shape (rows per warp x cells per lane), undoes them (the
 * state, clock and maxima are copied aside first), keeps the fastest shape and returns its
 * rows per warp in *rows_per_warp (nullable). */
hp2d_status hp2d_autotune(hp2d_ctx* ctx, int32_t trial_steps, int32_t* rows_per_warp);
/* Runs until the clock passes routing_time (or max_steps); returns steps executed. */
hp2d_status hp2d_run(hp2d_ctx* ctx, int64_t max_steps, int64_t* steps_done);

/* Failure handling of the fused path, the try/catch of HydroPol2D_Main_While.m:926-993.  A fused
 * step is rejected when a cell of finite elevation ends it with a non-finite depth or one below
 * -depth_tolerance, or when one of its row copies timed out.  A rejected step commits nothing:
 * depths, fluxes, soil storage and maxima stay those the step started from (d_t = d_p,
 * I_t = I_p), and so do the clock, counters and volumes.  A step rejected for its depths is
 * retried as the reference's catch block does: the clock goes back by the step, catch_index
 * grows, the new step is alfa_min*dx/sqrt(g*max(d_tot, d_p)) / catch_index / factor_reduction
 * (the last refresh's maximum velocity joins the celerity when flag_adaptive_timestepping = 0),
 * max_time_step drops to 1.5 x that step, and the rain interval is recomputed.  After
 * max_retries rejections of one step the call returns HP2D_NUMERICAL with the last accepted
 * state (defaults: 8 retries, factor_reduction 2 as input_data_script.m:486).  A timed-out step
 * is not retried: the call returns HP2D_TIMEOUT with the last accepted state.  With
 * dt_floor_is_error = 1 a step whose refreshed dt equals min_time_step (refreshing_timestep's
 * `unstable`, counted in hp2d_diag.unstable_steps either way) is kept and the call returns
 * HP2D_DT_FLOOR after it.  The velocity and hazard maxima keep what a rejected attempt added. */
hp2d_status hp2d_set_retry_policy(hp2d_ctx* ctx, int32_t max_retries, double factor_reduction,
                                  int32_t dt_floor_is_error);
/* Polls of one row-copy wait of the fused step before it gives up (default 4194304).  A copy
 * that has not landed then makes the step a rejected one and the call return HP2D_TIMEOUT;
 * copies still in flight are always waited for with the default limit before a block exits.
 * 0 makes every wait give up at once (a test of the timeout path). */
hp2d_status hp2d_set_wait_limit(hp2d_ctx* ctx, int64_t polls);
/* Test hook (no counterpart in the reference): the next `attempts` attempts of step k are
 * rejected as if a depth had gone non-finite, so that the retry path runs on demand. */
hp2d_status hp2d_inject_step_fault(hp2d_ctx* ctx, int64_t k, int32_t attempts);

/* ---- one grid in row slabs (one context per slab; no counterpart in the reference) ---- */
/* The context holds rows of a larger grid: its own rows [row0, row1) and up to two halo rows on
 * each side that neighbouring slabs own (the draining limiter's dependency radius).  Its fused
 * steps reduce the CFL maxima, the volume ledgers and the depth checks over the own rows only;
 * after every step the caller combines the slabs' maxima (hp2d_step_maxima: the ordered bits of
 * the largest speed^2 and wave-celerity term, and the next step's clamp skip), gives every slab
 * the combined values (hp2d_apply_refresh redoes the step's time-step refresh with them), and
 * copies each slab's two edge rows into its neighbours' halo rows (hp2d_copy_rows; the buffer is
 * host or device memory).  The slabs then step as one grid, bit for bit.  No infiltration, rain
 * maps, map records or retries in this mode (hydropol2d_b200.slabs drives it). */
hp2d_status hp2d_set_owned_rows(hp2d_ctx* ctx, int32_t row0, int32_t row1);
hp2d_status hp2d_step_maxima(hp2d_ctx* ctx, uint64_t* speed2_bits, uint64_t* celerity_bits, int32_t* clamp_skip);
hp2d_status hp2d_apply_refresh(hp2d_ctx* ctx, uint64_t speed2_bits, uint64_t celerity_bits, int32_t clamp_skip);
/* rows [row0, row0 + nrows) of the current state records ({h, q_x, q_y, dmax}, 4 values of the
 * context's precision per cell) to buffer (into_state = 0) or from it (1) */
hp2d_status hp2d_copy_rows(hp2d_ctx* ctx, int32_t row0, int32_t nrows, void* buffer, int32_t into_state);

/* Temporal blocking (no counterpart in the reference; opt-in): steps_per_block = K in 2..4 makes
 * hp2d_fused_steps advance K steps per launch at the time step of the last refresh, which then
 * runs only on step 1 and on the steps k with (k - 1) % K == 0 (refreshing_timestep.m:17-368
 * runs every step in the reference, so results follow the frozen-step schedule, not the per-step
 * one).  Each block stages 64 x 32 output cells with a 2K-cell halo in shared memory by TMA and
 * writes them back once.  Steps that do not fill an aligned block, and blocks in which an outlet
 * cell asked for the clamp skip of Hydrological_Model.m:45-50 or a step was rejected, run one
 * per launch under the same schedule.  FP32 only; no rain, infiltration, inflow, stage, control
 * structures, map records or hazard maps (HP2D_UNSUPPORTED_FLAG at the next fused call); the
 * dry-row skips are off while it is on.  steps_per_block = 1 switches it off; 0 lets
 * hp2d_autotune choose K among 1..4 by measured time per step. */
hp2d_status hp2d_set_temporal_blocking(hp2d_ctx* ctx, int32_t steps_per_block);

/* ---- outputs ---------------------------------------------------------------------- */
hp2d_status hp2d_download(hp2d_ctx* ctx, int32_t field, double* host, size_t count);
/* Raw copy of an internal array in the context's precision and SI units, for callers
 * that keep the state in their own units (and for bit-level regression checks):
 *   0 depth [m], 1 right-face discharge per width [m^2/s], 2 upper-face discharge
 *   [m^2/s], 3 soil storage [m], 4 recovery timer [s], 5 dmax [m], 6 arrival [s],
 *   7 Hf x [m], 8 Hf y [m] (after hp2d_li_step), 9 Hf at outlets [m] and 10 outlet
 *   sink rate [m/s] (one value per outlet cell, in increasing linear-index order).
 * `bytes` must equal the array size exactly. */
hp2d_status hp2d_download_native(hp2d_ctx* ctx, int32_t field, void* host, size_t bytes);
hp2d_status hp2d_get_diag(hp2d_ctx* ctx, hp2d_diag* out);
/* Stored surface volume sum(d_t)*cell_area/1000 [m^3], FP64 accumulation. */
hp2d_status hp2d_stored_volume(hp2d_ctx* ctx, double* volume);

/* ---- batched ensemble ------------------------------------------------------------- */
/* Replaces the member loop of HydroPol2D_Main_While_Ensemble.m:46-139 (and the per-member
 * runs of Probabilistic_dam_break_analysis.m:8-60), which call the surface-flow step once
 * per member in turn.  Members are ordinary FP32 contexts, each set up with the calls
 * above (own grid size, DEM, roughness, rain or initial state, clock and dt); the ensemble
 * advances every member that has not reached its routing_time by one of its own steps per
 * launch: one persistent kernel whose CTAs take (member, block of rows) items from a
 * queue, with each member's dt refresh and clock advance done by the CTA that completes
 * its last item.  Members must agree on Green-Ampt on/off and on uniform vs map rain.
 * While in an ensemble a member must not be stepped on its own concurrently; its
 * outputs are read with hp2d_download / hp2d_get_diag as usual. */
typedef struct hp2d_ensemble hp2d_ensemble;
hp2d_status hp2d_ensemble_create(int32_t device, hp2d_ensemble** out);
hp2d_status hp2d_ensemble_destroy(hp2d_ensemble* ens);
const char* hp2d_ensemble_last_error(const hp2d_ensemble* ens);
hp2d_status hp2d_ensemble_add(hp2d_ensemble* ens, hp2d_ctx* member);
/* rows each warp streams (>= 4) and cells per lane (1 or 2) for every member;
 * hp2d_ensemble_autotune picks both */
hp2d_status hp2d_ensemble_set_tuning(hp2d_ensemble* ens, int32_t rows_per_warp);
hp2d_status hp2d_ensemble_set_layout(hp2d_ensemble* ens, int32_t cells_per_lane);
hp2d_status hp2d_ensemble_autotune(hp2d_ensemble* ens, int32_t trial_steps, int32_t* rows_per_warp);
/* nsteps launches; *n_active (nullable) = members still running afterwards */
hp2d_status hp2d_ensemble_steps(hp2d_ensemble* ens, int32_t nsteps, int32_t* n_active);
hp2d_status hp2d_ensemble_steps_timed(hp2d_ensemble* ens, int32_t nsteps, int32_t* n_active,
                                      float* elapsed_ms);
/* until every member has reached its routing_time (or max_steps launches, if > 0) */
hp2d_status hp2d_ensemble_run(hp2d_ensemble* ens, int64_t max_steps, int64_t* steps_done);

/* ---- allocation-free timestep (no counterpart in the reference) -------------------- */
/* refreshing_timestep's refresh branch (as hp2d_cfl_dt) on caller-owned FP32 device
 * arrays, for callers that may not allocate GPU memory while they run: a MEX gateway
 * inside MATLAB whose GPU memory pool owns the device, real-time drivers that allocate
 * only at start-up.  Nothing is allocated: the reduction
 * scratch is a fixed 64 KB array inside the library, resident on every GPU that loads it
 * until the process exits, which limits grids to ny <= 65536 rows (larger grids are
 * rejected with HP2D_INVALID_ARG).  The first call on each device (with that device
 * current) resolves the array's device address and should come before any stream
 * capture.  Calls that overlap on the GPU share the scratch and race.
 *   q_x, q_y   ny*nx limited face discharge per unit width [m^2/s] (native fields 1, 2)
 *   hf         3*ny*nx face flow depth [m]: pages x, y and outlet, as Hf(:,:,1:3)
 *   stream     cudaStream_t to run on (NULL = default stream); the call ends by copying
 *              the two maxima to host memory and synchronising this stream, so a stream
 *              under capture is refused with HP2D_INVALID_ARG (nothing enters the capture)
 *   time_step  [out] new time step [min]; max_velocity [out, nullable] [m/s]
 * On failure hp2d_noalloc_error() gives the message. */
hp2d_status hp2d_cfl_dt_noalloc(int32_t ny, int32_t nx, double resolution, const hp2d_params* params,
                                const float* q_x, const float* q_y, const float* hf, void* stream,
                                double* time_step, double* max_velocity);
const char* hp2d_noalloc_error(void);

#ifdef __cplusplus
}
#endif

#endif /* HP2D_H */
