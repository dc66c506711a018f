/* ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of n2p2's 2G-HDNNP prediction path, used by the tests
 * (and smoke check) as an independent CPU checker of the CUDA path.  It
 * follows the reference's per-symmetry-function code path (SymFnc*::calculate,
 * not the grouped SymGrp* path the CUDA kernels restate), so agreement with
 * both is a cross-check of the grouping.  Pinned against the reference's
 * golden vectors (test/cpp/ExamplePrediction.h) by tests/test_oracle_golden.py.
 */
#ifndef HDNNP_ORACLE_H
#define HDNNP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define HO_MAX_ELEM 8
#define HO_MAX_LAYERS 8

typedef struct
{
    int    type;          /* 2, 3, 9 */
    int    e1, e2;        /* neighbor elements (e2 unused for type 2) */
    double eta, rs, rc, zeta, lambda;
    int    zetaInt, useIntegerPow;
    int    scalingType;   /* 0 none, 1 scale, 2 center, 3 scalecenter, 4 sigma */
    double Smin, Gmin, Gmean, scalingFactor;
    int    slot[HO_MAX_ELEM];  /* dG/dr slot per neighbor element, -1 none */
} ho_sf;

typedef struct
{
    int           numElements;
    int           cutoffType;
    double        cutoffAlpha;
    int           numSF[HO_MAX_ELEM];
    ho_sf const*  sfs[HO_MAX_ELEM];     /* sorted (NN input order) */
    int           numSlots[HO_MAX_ELEM][HO_MAX_ELEM];
    int           numLayers[HO_MAX_ELEM];
    int           neurons[HO_MAX_ELEM][HO_MAX_LAYERS];
    int           activation[HO_MAX_ELEM][HO_MAX_LAYERS];
    double const* connections[HO_MAX_ELEM];  /* setConnections order */
    int           normalizeNeurons;
    int           normalize;
    double        meanEnergy, convEnergy, convLength;
    double        atomEnergy[HO_MAX_ELEM];
} ho_potential;

/* Prediction::readStructureFromFile + Prediction::predict on arrays.
 * box: 9 doubles (rows = lattice vectors) or NULL.  Returns 0 on success.
 * energy: physical units with offsets; forces: n x 3; atomic_energies
 * (nullable): per-atom NN energies in physical units. */
int ho_predict(ho_potential const* P, int n, double const* box,
               double const* pos, int const* elem, double* energy,
               double* forces, double* atomic_energies);

/* CutoffFunction::fdf for cutoff `type` (n2p2 numbering), radius rc and
 * inner fraction alpha. */
void ho_cutoff_fdf(int type, double rc, double alpha, double r, double* fc,
                   double* dfc);

/* Neighbor counts / list after the last ho_predict call's neighbor search
 * (reference order); index may be NULL to query the total only. */
long ho_last_num_entries(void);
void ho_last_neighbors(long* counts, long* index, double* dr, double* d);
/* Scaled symmetry functions of the last call, [atom][stride]. */
void ho_last_G(double* G, int stride);

#ifdef __cplusplus
}
#endif

#endif
