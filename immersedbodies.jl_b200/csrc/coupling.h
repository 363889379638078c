// coupling.h -- launchers of the coupling kernels (coupling.cu, built with -fmad=false).
#pragma once
#include "common.cuh"

namespace ibpm {

constexpr int kTile = 16;  // faces per side of a reg! gather tile

void launch_reg_weights(const Panels &P, int p0, int p1, const Grid &g, cudaStream_t st);
void launch_bbox(const Panels &P, const Grid &g, cudaStream_t st);
// reg! onto a patch of element type T (double or float); forces f are double.
template <class T>
void launch_reg_patch(const Panels &P, const double *f, long long fbs, T *patch, long long pbs, int nbatch,
                      const Grid &g, cudaStream_t st);
// regT! from a level-1 flux of element type T, summed in double.
template <class T>
void launch_regT(const Panels &P, const T *q, long long qbs, double *out, long long obs, int nbatch, int add_q0,
                 const StepDev *prm, const Grid &g, cudaStream_t st);
// The same for the cases of a batched ensemble group (tab: ncase device
// CaseViews): each case's E^T F~b onto its patch, and each case's
// Ftmp = E (qs + q0) - ub h from its flux slot (q + case qbs) and prm[case].
template <class T>
void launch_reg_patch_multi(const CaseView *tab, int ncase, const Grid &g, cudaStream_t st);
template <class T>
void launch_regT_multi(const CaseView *tab, int ncase, int np_max, const T *q, long long qbs, const StepDev *prm,
                       const Grid &g, cudaStream_t st);
void launch_rigid_motion(const Panels &P, const double *ref_xb, const double *motion, int p0, int p1,
                         cudaStream_t st);

}  // namespace ibpm
