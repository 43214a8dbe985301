// rc_host.h -- host-side data of the solver: validated parameters, multigrid
// geometry and spectral tables.  No CUDA in here; rc_context.cu uploads
// these to the device.
#pragma once
#include <stdint.h>
#include <string>
#include <vector>
#include "radchan.h"

namespace rc_detail {
// message of the last failure of a context-free call (per host thread)
inline thread_local std::string g_err;

inline int set_err(std::string *dst, int code, const std::string &m) {
    if (dst) *dst = m;
    g_err = m;
    return code;
}
}  // namespace rc_detail

namespace rc {

// Wall treatment used by the march; derived from param.h bd* and the
// adiabatic flags (mc_gpu_noint.cu:375-654).
enum WallType : int {
    WT_PERIODIC = 1,     // bd = 1
    WT_BLACK_FIXED = 2,  // bd = 2, emits I_b(Tw) of the wall
    WT_SPECULAR = 3,     // bd = 3 (reflection done correctly on every axis)
    WT_BLACK_CELL = 4,   // bd = 4, emits I_b of the first interior cell
    WT_LOST = 5,         // bd = 5, bundle discarded
    WT_BLACK_FACE = 6,   // bd = 2 with adiabatic flag: I_b of the face average
};

// One multigrid level (definitions.h:60-136).
struct GridLevel {
    int im = 0, jm = 0, km = 0, maxs = 0;
    std::vector<float> xu, yu, zu;  // faces: im+1, jm+1, km+1
    std::vector<float> x, y, z;     // centres with ghosts: im+2, jm+2, km+2
};

void build_grid_level(const rc_params &p, int level, GridLevel &g);

// Host copy of one spectral table set, in the reference's layouts.
struct TableSet {
    int nT = 0, nB = 0, nQ = 0;
    std::vector<float> Tnb, kP, kR, kM;   // [nT] (kR, kM only carried for the file format)
    std::vector<float> wvl, wvr, wvc;     // [nB]
    std::vector<float> kavg;              // [nB]
    std::vector<float> kavg_t;            // [nT][nB] band-mean k per temperature row
    std::vector<float> kq;                // [nB][nT][nQ]
    std::vector<float> prob;              // [nT][nB]
    std::vector<float> probg;             // [nT][nB][nQ]
    std::vector<float> wq, gq;            // [nQ]
    void view(rc_tables *t) const;
    void from_view(const rc_tables *t);
};

int tables_synthetic(const rc_synth_spec &s, TableSet &out, std::string &err);
int tables_read_dir(const std::string &dir, int nT, int nB, int nQ, TableSet &out, std::string &err);
int tables_write_dir(const TableSet &ts, const std::string &dir, std::string &err);
// What the device lookups assume of a table set: 2..256 increasing,
// uniformly spaced temperatures; cumulative probabilities finite,
// non-decreasing, within [0, 1]; absorption coefficients and the
// Planck-mean coefficient finite and >= 0.  RC_E_INVALID and a message
// naming the first violation otherwise.
int tables_check(const TableSet &t, std::string &err);

// Host copy of a particle scattering table set (rc_scattering layouts).
struct ScatterSet {
    int nB = 0, nQ = 0, nA = 0;
    std::vector<float> wvl, wvr, wvc;   // [nB] band edges and centres (0 when synthetic)
    std::vector<float> kabs, ksca;      // [nB][nQ]
    std::vector<float> theta;           // [nA] radians
    std::vector<float> cdf;             // [nB][nA]
    void view(rc_scattering *s) const;
};

int scattering_synthetic(const rc_scatter_spec &spec, ScatterSet &out, std::string &err);
int scattering_read_dir(const std::string &dir, int nB, int nQ, ScatterSet &out, std::string &err);
int scattering_write_dir(const ScatterSet &s, const std::string &dir, std::string &err);
// The checks of rc_scattering_validate.
int scattering_check(const rc_scattering &s, std::string &err);

// Gauss-Legendre nodes/weights on [-1, 1] (Newton iteration on P_n).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w);

int params_default(rc_params &p);
int params_from_headers(const std::string &param_h, const std::string &nb_h, rc_params &p, std::string &err);
int params_validate(const rc_params &p, std::string &err);
void wall_types(const rc_params &p, int wt[6]);

// Deterministic double uniform in [0,1) from the Philox stream (seed, stream, idx).
double synth_uniform(uint64_t seed, uint32_t stream, uint32_t idx);

}  // namespace rc

// Opaque handles of the C ABI.
struct rc_table_set {
    rc::TableSet ts;
};
struct rc_scatter_set {
    rc::ScatterSet s;
};
