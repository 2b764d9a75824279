// Internal data model of the B200 flow solver (shared by host and device code).
//
// HBM layout (all structure-of-arrays, int32 indices):
//   faces  : fc0[F], fc1[F] cell ids in the reference's roles (cell0 < cell1);
//            a boundary face has fc1 = N + side, so fc1 indexes the field's
//            boundary slot directly.  Geometry area/lam/rl/S/xf per face.
//   cells  : nbr[6][N]   neighbour through slot f (cell_faces order), or
//                        -1 - face for a boundary face;
//            sface[6][N] the cell's faces sorted by reference face id (the
//                        order in which the reference's face loops touch the cell);
//            xc/yc/zc, vol, rho.
//   fields : U V W P PP T, each N + 6 doubles (interior, then 6 boundary slots);
//            gradients grad[field][component][N].
//   systems: 7-point rows stored ELL-style: diag[N], off[6][N], col[6][N]
//            (slot k = the cell's k-th face in sorted order; boundary slots
//            have col = row and value 0).
#pragma once

#include <stdint.h>

namespace mcb {

enum Side { FRONT = 0, BACK = 1, LEFT = 2, RIGHT = 3, DOWN = 4, UP = 5 };
enum BoundaryType { WALL = 1, INLET = 2, OUTLET = 3 };
enum GradField { G_U = 0, G_V = 1, G_W = 2, G_P = 3, G_PP = 4, G_T = 5, G_NFIELDS = 6 };

struct DeviceMesh {
    int N = 0, F = 0;
    int *fc0 = nullptr, *fc1 = nullptr;
    int *nbr = nullptr;     // [6][N]
    int *sface = nullptr;   // [6][N]
    int *col = nullptr;     // [6][N] ELL columns, sorted-face slot order
    double *area = nullptr, *lam = nullptr, *rl = nullptr;
    double *Sx = nullptr, *Sy = nullptr, *Sz = nullptr;
    double *xf = nullptr, *yf = nullptr, *zf = nullptr;
    double *xc = nullptr, *yc = nullptr, *zc = nullptr;
    double *vol = nullptr, *rho = nullptr;
    int *outlet_faces = nullptr;  // list of outlet faces
    int n_outlet = 0;
};

// Scalars shared by the physics kernels (passed by value).
struct Physics {
    int N;
    int mode;             // 0 compat, 1 simple
    int btype[6];
    int last_bface[6];    // last face (reference order) of each boundary side
    int cell0;            // the handle's id of the reference's cell 0
    double mu, inlet_mu, u_in, rho_in, T_ref, rdelta;
    double urf_u, urf_T, urf_p, flux_corr;
    // scalar transports: inlet value per scalar type (SC_*), computed on the
    // host as the reference computes it (FlowSolver.inl:2625-2659), and
    // Cmu^0.75 of the k-epsilon wall functions (:2786, :2834)
    double sc_inlet[7];
    double cmu75;
};

// Scalar types of Scalar_solve (the reference's utils.hpp:31-37).
enum ScalarType { SC_TERBTE = 0, SC_TERBED = 1, SC_TEMP = 2, SC_FUEL = 3, SC_PROG = 4, SC_VARFU = 5, SC_VARPR = 6 };

// Balance of boundary fluxes (calculate_mass_flux, FlowSolver.inl:2010-2079).
struct FluxBalance {
    double flow_in, flow_out, area_out;
    double outlet_scale;  // simple mode: multiply outlet fluxes
    double rate_area;     // fallback when flow_out < 1e-10
    int fallback;
    int pad;
};

} // namespace mcb
