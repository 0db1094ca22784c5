/* oracle/bz_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the algorithms on the Barnes-Hut / TreePM gravity path, used to check
 * the CUDA library (tests, smoke(), bench.py's CPU baseline).  Never linked into the
 * product.  Parity is pinned: the restated reference pieces (or_morton_ref,
 * or_ref_linear_octree, or_ref_walk, or_pm_periodic, or_fp64_pairwise) are checked against
 * the reference's own code compiled from its sources (oracle/_ref) and against the golden
 * fixtures under tests/golden/ generated from it.
 *
 * Conventions: positions/masses are FP32 as in the reference particle layout
 * (engine/physics/core/particle/PhyParticleSoAView.hpp:18-33); accumulation is FP64.
 */
#ifndef BZ_ORACLE_H
#define BZ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Morton keys --------------------------------------------------------------------- */
void or_bbox_f32(const float* x, const float* y, const float* z, int64_t n, float out6[6]);
void or_morton_ref(const float* x, const float* y, const float* z, int64_t n,
                   const float bbox6[6], int fused, uint64_t* keys);
void or_morton63(const double* x, const double* y, const double* z, int64_t n,
                 const double origin3[3], double size, uint64_t* keys);
void or_stable_sort_u64(const uint64_t* keys, int64_t n, int32_t* perm);

/* ---- reference linear octree (compat topology) ---------------------------------------- */
/* fused: evaluate the reference's multiply-add expressions as fused (its CUDA build) or not
 * (its sources compiled for the host). */
int64_t or_ref_linear_octree(const float* x, const float* y, const float* z, const float* m,
                             int64_t n, int leaf_capacity, int fused, int64_t node_cap,
                             float* hot8, int32_t* next, int32_t* child_mask,
                             int32_t* first_child, int32_t* leaf_start, int32_t* leaf_count,
                             uint64_t* sorted_keys, int32_t* sorted_index, int32_t* leaf_depth);
void or_ref_walk(const float* x, const float* y, const float* z, const float* m, int64_t n,
                 const float* hot8, const int32_t* next, const int32_t* child_mask,
                 const int32_t* first_child, const int32_t* leaf_start,
                 const int32_t* leaf_count, const int32_t* sorted_index, int32_t root,
                 float theta, float softening, float min_distance2, float max_acceleration,
                 int criterion, float split_scale, float cutoff2, double* acc3);

/* ---- production adaptive octree -------------------------------------------------------- */
int64_t or_build_tree(const uint64_t* skeys, const float* pos4, int64_t n, int leaf_cap,
                      int max_level, int64_t node_cap, int32_t* start, int32_t* count,
                      int32_t* child, int32_t* nchild, int32_t* parent, int32_t* level,
                      float* mono4, float* bmin3, float* bmax3, float* quad6);

typedef struct {
    float theta2;    /* theta*theta, rounded to FP32 */
    float eps2;      /* softening^2 */
    float rcut2;     /* 0 disables the cutoff */
    float box;       /* periodic box length; 0 = open boundaries */
    float rsplit;    /* Gaussian split scale r_s; 0 = Newtonian */
    float min_dist2; /* pairs with softened r^2 <= this are skipped */
    int quadrupole;  /* 1 = monopole + quadrupole for accepted nodes */
    int group;       /* targets per group (32) */
    float max_node_size; /* > 0: nodes with extent >= this are never accepted */
} or_walk_params;

int64_t or_tree_groups(const int32_t* start, const int32_t* count, const int32_t* child,
                       const int32_t* nchild, const float* bmin3, const float* bmax3,
                       const float* mono4, int32_t gmax, int64_t* gstart);
/* gstart == NULL: fixed groups of prm->group consecutive targets; else ngroups tree groups
 * given by or_tree_groups. */
void or_walk(const float* pos4, int64_t n, const int32_t* start, const int32_t* count,
             const int32_t* child, const int32_t* nchild, const float* mono4,
             const float* bmin3, const float* bmax3, const float* quad6,
             const or_walk_params* prm, const int64_t* gstart, int64_t ngroups, double* acc3,
             double* pot, int64_t* n_pp, int64_t* n_pn);
/* As or_walk for the groups only[0..n_only) (NULL: all); asum (may be NULL) receives, per
 * target, the sum of the magnitudes of its pair and node terms. */
void or_walk_ex(const float* pos4, int64_t n, const int32_t* start, const int32_t* count,
                const int32_t* child, const int32_t* nchild, const float* mono4,
                const float* bmin3, const float* bmax3, const float* quad6,
                const or_walk_params* prm, const int64_t* gstart, int64_t ngroups, double* acc3,
                double* pot, int64_t* n_pp, int64_t* n_pn, const int64_t* only, int64_t n_only,
                double* asum);

/* ---- direct sums --------------------------------------------------------------------- */
void or_direct_f64(const float* pos4, int64_t n, const int64_t* targets, int64_t nt,
                   double eps, double box, double rsplit, double rcut, double* acc3,
                   double* pot);
void or_ewald_f64(const float* pos4, int64_t n, const int64_t* targets, int64_t nt, double eps,
                  double box, double alpha, int kmax, double* acc3);

/* ---- periodic particle-mesh leg ------------------------------------------------------- */
void or_fft3d(double* re_im, int size, int inverse);
int or_pm_periodic(const float* pos4, int64_t n, int mesh, double box, double rsplit, int order,
                   int gradient, double floor_w, double* acc3, double* density, double* phi);
/* The same mesh, interpolated only at targets[0..nt) (all particles when NULL). */
int or_pm_periodic_at(const float* pos4, int64_t n, int mesh, double box, double rsplit,
                      int order, int gradient, double floor_w, const int64_t* targets, int64_t nt,
                      double* acc3, double* density, double* phi);

/* Isolated PM of the reference's GPU TreePM (doubled mesh of 2 grid_half cells). */
int or_pm_isolated(const float* pos4, int64_t n, int grid_half, float cell_floor, float softening,
                   double rsplit_cells, int order, int gradient, double floor_w,
                   const int64_t* targets, int64_t nt, double* acc3, double* params8,
                   double* density, double* phi_out);

/* ---- split kernel helpers ---------------------------------------------------------------- */
double or_split_weight(double s, double rsplit);

/* ---- learned pair correction (MLP with the engine's BF16 rounding points) ---------- */
void or_mlp_forward(const float* params, const float* x6, int64_t n, float scale, float* out3);
void or_mlp_grad(const float* params, const float* x6, const float* y3, int64_t n, double* grad,
                 double* loss);

#ifdef __cplusplus
}
#endif
#endif
