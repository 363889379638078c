// warmstart.h -- internal interface between the solver engine (ibpm.cu) and the
// learned CG warm start (warmstart.cu).
//
// The warm start improves the moving-body force solve's initial guess
// (src/coupling.jl:194-202 starts cg! from the previous F~b).  Per step: a
// Galerkin step in the B-energy norm along the last change of the solution
// gives x_e; the network maps the residual b - B x_e (with context) to a
// correction p, an approximate B^-1 (b - B x_e); a second Galerkin step along p
// gives the guess.  Plain CG then runs to the configured tolerance from it.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "../../include/ibpm_b200.h"

namespace ibpm {

// Feature channels per body point (the network's input width).
//   0, 1  r / |r|, r = b - B x_e the residual of the extrapolated guess x_e (x, y)
//   2, 3  F1, the previous step's solution F~b (x, y)
//   4, 5  d / |d|, d = F1 - F2 its last change (x, y)
//   6, 7  ub, the body-point velocity (x, y)
//   8, 9  cos(angle), sin(angle) of the point's body
// |v| is the RMS of v over the sample's 2 np entries, so every step is a
// unit-size example of the same (linear) map from residual to error.
constexpr int kWsFeatures = 10;
constexpr int kWsOutputs = 2;

// feat[c * np + p] for the channels above (bx = B x_e); vectors of length 2 np
// are stored x block then y block, ub is np x 2 column-major, motion is
// nbody x 6 (angle at 4); scale[0] <- |r|.
void launch_ws_features(const double *ftmp, const double *bx, const double *f1, const double *d, const double *ub,
                        const double *motion, const int *pbody, int np, float *feat, double *scale, cudaStream_t st);
// z = [f1 | d] in blocks of 2 np, d = f1 - f2; then f2 <- f1.
void launch_ws_direction(const double *f1, double *f2, int np, double *z, cudaStream_t st);
// p = out_mean + out_std * y, the network's output in solver units.
void launch_ws_prediction(const float *y, const ibpm_net *net, int np, double *p, cudaStream_t st);
// Galerkin step in the B-energy norm over the k = 1 or 2 directions of
// z = [x | v_1 .. v_k] (bz = B z): x_out <- x + sum y_i v_i with y minimising
// the energy norm of the error over that span, c <- B x_out; x2, c2 (optional)
// receive copies and coef (optional) the first coefficient y_1.
void launch_ws_galerkin(const double *z, const double *bz, const double *b, double *x, double *c, double *x2,
                        double *c2, int np, int k, double *coef, cudaStream_t st);

// Projection onto previous solutions: V = [v_0 .. v_(k-1)] (k <= 16, most recent
// first, zero vectors allowed), BV = B V, vectors of n doubles.  x <- the
// combination of V minimising the B-energy norm of the error (Galerkin over
// span V, with near-dependent directions dropped), c <- B x; G (k x k), h (k)
// are scratch; kept (optional) receives the number of directions used.
void launch_ws_projection(const double *V, const double *BV, const double *b, double *x, double *c, int n, int k,
                          double *G, double *h, double *kept, cudaStream_t st);
// hist[j] <- hist[j-1] (j = k-1 .. 1), hist[0] <- f.
void launch_ws_shift(double *hist, const double *f, int n, int k, cudaStream_t st);

// Floats of activation scratch a forward pass of batch B over n points needs.
size_t net_act_floats(const ibpm_net *net, int B, int n);
// Forward pass on the device on stream st: x [B][cin][n] (raw features,
// normalised inside) -> y [B][cout][n] (normalised outputs).
void net_forward_dev(const ibpm_net *net, const float *x, int B, int n, float *act, float *y, cudaStream_t st);
int net_device(const ibpm_net *net);
int net_cin(const ibpm_net *net);
int net_cout(const ibpm_net *net);

}  // namespace ibpm
