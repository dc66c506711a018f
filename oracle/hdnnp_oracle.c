/* ORACLE / TEST INFRASTRUCTURE ONLY -- see hdnnp_oracle.h.
 *
 * Plain C99 restatement of the reference's prediction path, compiled with
 * -ffp-contract=off (the reference's ISO C++ build does not contract).
 * Each function names the reference code it restates.
 */
#include "hdnnp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct
{
    long    index;
    int     element;
    double  d;
    double  dr[3];
    double* dGdr;  /* [numSlots(ec, element)][3] */
} ho_nbr;

typedef struct
{
    int     element;
    double  r[3];
    int     numSF;
    long    numNbr;
    long    capNbr;
    ho_nbr* nbr;
    double* G;
    double* dEdG;
    double* dGdrSelf;  /* [numSF][3] */
    double  energy;
    double  f[3];
} ho_atom;

static ho_atom* g_atoms = NULL;
static int      g_n = 0;
static int      g_maxSF = 0;

static void ho_free_atoms(void)
{
    for (int i = 0; i < g_n; ++i)
    {
        for (long k = 0; k < g_atoms[i].numNbr; ++k) free(g_atoms[i].nbr[k].dGdr);
        free(g_atoms[i].nbr);
        free(g_atoms[i].G);
        free(g_atoms[i].dEdG);
        free(g_atoms[i].dGdrSelf);
    }
    free(g_atoms);
    g_atoms = NULL;
    g_n = 0;
}

/* ---- CutoffFunction::fdf (libnnp/CutoffFunction.h:210-220,
 *      CutoffFunction.cpp:128-213; CoreFunction.h:171-320) ---------------- */
typedef struct
{
    int    type;
    double rc, rcinv, rci, iw;
} ho_cutoff;

/* CutoffFunction::PI, CoreFunction::E, CutoffFunction::TANH_PRE, made as
 * the reference makes them (libnnp/CutoffFunction.cpp:24-27). */
static double ho_PI, ho_E, ho_TANH_PRE;

static void ho_constants(void)
{
    ho_PI = 4.0 * atan(1.0);
    ho_E = exp(1.0);
    ho_TANH_PRE = pow((ho_E + 1 / ho_E) / (ho_E - 1 / ho_E), 3);
}

static ho_cutoff ho_make_cutoff(int type, double rc, double alpha)
{
    ho_cutoff c;
    c.type = type;
    c.rc = rc;
    c.rcinv = 1.0 / rc;
    c.rci = rc * alpha;
    c.iw = 1.0 / (rc - c.rci);
    return c;
}

static void ho_fdf(ho_cutoff const* c, double r, double* fc, double* dfc)
{
    if (r >= c->rc) { *fc = 0.0; *dfc = 0.0; return; }
    if (c->type == 0) { *fc = 1.0; *dfc = 0.0; return; }           /* HARD */
    if (c->type == 2 || c->type == 3)                              /* TANHU/TANH */
    {
        double const t = tanh(1.0 - r * c->rcinv);
        double const t2 = t * t;
        if (c->type == 2)
        {
            *fc = t * t2;
            *dfc = 3.0 * t2 * (t2 - 1.0) * c->rcinv;
        }
        else
        {
            *fc = ho_TANH_PRE * t * t2;
            *dfc = 3.0 * ho_TANH_PRE * t2 * (t2 - 1.0) * c->rcinv;
        }
        return;
    }
    if (r < c->rci) { *fc = 1.0; *dfc = 0.0; return; }
    double const x = (r - c->rci) * c->iw;
    if (c->type == 1)                                              /* COS */
    {
        double const t = cos(ho_PI * x);
        *fc = 0.5 * (t + 1.0);
        *dfc = -0.5 * c->iw * ho_PI * sqrt(1.0 - t * t);
        return;
    }
    double fx, dfx;
    switch (c->type)
    {
    case 4: /* EXP */
    {
        double const t = 1.0 / (x * x - 1.0);
        double const t2 = exp(t);
        fx = ho_E * t2;
        dfx = -2.0 * ho_E * x * t * t * t2;
        break;
    }
    case 5: /* POLY1 */
        fx = (2.0 * x - 3.0) * x * x + 1.0;
        dfx = x * (6.0 * x - 6.0);
        break;
    case 6: /* POLY2 */
    {
        double const x2 = x * x;
        fx = ((15.0 - 6.0 * x) * x - 10.0) * x * x2 + 1.0;
        dfx = x2 * ((60.0 - 30.0 * x) * x - 30.0);
        break;
    }
    case 7: /* POLY3 */
    {
        double const x2 = x * x;
        fx = (x * (x * (20.0 * x - 70.0) + 84.0) - 35.0) * x2 * x2 + 1.0;
        dfx = x2 * x * (x * (x * (140.0 * x - 420.0) + 420.0) - 140.0);
        break;
    }
    default: /* POLY4 */
    {
        double x4 = x * x;
        x4 *= x4;
        fx = (x * (x * ((315.0 - 70.0 * x) * x - 540.0) + 420.0) - 126.0)
             * x * x4 + 1.0;
        dfx = x4 * (x * (x * ((2520.0 - 630.0 * x) * x - 3780.0) + 2520.0)
                    - 630.0);
        break;
    }
    }
    *fc = fx;
    *dfc = dfx * c->iw;
}

/* utility.cpp:292-317 pow_int */
static double ho_pow_int(double x, int n)
{
    unsigned m;
    if (n < 0) { x = 1.0 / x; m = (unsigned)(-n); }
    else m = (unsigned)n;
    double result = 1.0;
    do
    {
        if (m & 1u) result *= x;
        m >>= 1;
        x *= x;
    }
    while (m);
    return result;
}

/* SymFnc::scale (libnnp/SymFnc.cpp:150-174) */
static double ho_scale(ho_sf const* s, double v)
{
    switch (s->scalingType)
    {
    case 0: return v;
    case 1: return s->Smin + s->scalingFactor * (v - s->Gmin);
    case 2: return v - s->Gmean;
    case 3: return s->Smin + s->scalingFactor * (v - s->Gmean);
    case 4: return s->Smin + s->scalingFactor * (v - s->Gmean);
    default: return 0.0;
    }
}

/* ---- Structure: inverse box, remap, pbc copies, neighbor list ---------- */

static void ho_inverse_box(double const b[3][3], double inv[3][3])
{
    /* Structure::calculateInverseBox (libnnp/Structure.cpp:519-546) */
    double invdet = b[0][0] * b[1][1] * b[2][2] + b[1][0] * b[2][1] * b[0][2]
                  + b[2][0] * b[0][1] * b[1][2] - b[2][0] * b[1][1] * b[0][2]
                  - b[0][0] * b[2][1] * b[1][2] - b[1][0] * b[0][1] * b[2][2];
    invdet = 1.0 / invdet;
    inv[0][0] = b[1][1] * b[2][2] - b[2][1] * b[1][2];
    inv[0][1] = b[2][1] * b[0][2] - b[0][1] * b[2][2];
    inv[0][2] = b[0][1] * b[1][2] - b[1][1] * b[0][2];
    inv[1][0] = b[2][0] * b[1][2] - b[1][0] * b[2][2];
    inv[1][1] = b[0][0] * b[2][2] - b[2][0] * b[0][2];
    inv[1][2] = b[1][0] * b[0][2] - b[0][0] * b[1][2];
    inv[2][0] = b[1][0] * b[2][1] - b[2][0] * b[1][1];
    inv[2][1] = b[2][0] * b[0][1] - b[0][0] * b[2][1];
    inv[2][2] = b[0][0] * b[1][1] - b[1][0] * b[0][1];
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c) inv[k][c] *= invdet;
}

static void ho_remap(double r[3], double const b[3][3], double const inv[3][3])
{
    /* Structure::remap (libnnp/Structure.cpp:1223-1247) */
    double f[3];
    for (int k = 0; k < 3; ++k)
        f[k] = r[0] * inv[0][k] + r[1] * inv[1][k] + r[2] * inv[2][k];
    for (int k = 0; k < 3; ++k) if (f[k] > 1.0) f[k] -= (int)f[k];
    for (int k = 0; k < 3; ++k) if (f[k] < 0.0) f[k] += 1.0 - (int)f[k];
    for (int k = 0; k < 3; ++k) if (f[k] == 1.0) f[k] = 0.0;
    for (int k = 0; k < 3; ++k)
        r[k] = f[0] * b[0][k] + f[1] * b[1][k] + f[2] * b[2][k];
}

static void ho_cross(double const a[3], double const b[3], double w[3])
{
    w[0] = a[1] * b[2] - a[2] * b[1];
    w[1] = a[2] * b[0] - a[0] * b[2];
    w[2] = a[0] * b[1] - a[1] * b[0];
}

static void ho_normalize(double v[3])
{
    double const n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= n;
    v[1] /= n;
    v[2] /= n;
}

static void ho_pbc_copies(double const b[3][3], double rc, int pbc[3])
{
    /* Structure::calculatePbcCopies (libnnp/Structure.cpp:486-517) */
    double axb[3], axc[3], bxc[3];
    ho_cross(b[0], b[1], axb);
    ho_normalize(axb);
    ho_cross(b[0], b[2], axc);
    ho_normalize(axc);
    ho_cross(b[1], b[2], bxc);
    ho_normalize(bxc);
    double const proj[3] = {
        fabs(b[0][0] * bxc[0] + b[0][1] * bxc[1] + b[0][2] * bxc[2]),
        fabs(b[1][0] * axc[0] + b[1][1] * axc[1] + b[1][2] * axc[2]),
        fabs(b[2][0] * axb[0] + b[2][1] * axb[1] + b[2][2] * axb[2])};
    for (int k = 0; k < 3; ++k)
    {
        pbc[k] = 0;
        while (pbc[k] * proj[k] <= rc) pbc[k]++;
    }
}

static void ho_push_nbr(ho_atom* a, long j, int el, double const dr[3])
{
    if (a->numNbr == a->capNbr)
    {
        a->capNbr = a->capNbr ? 2 * a->capNbr : 64;
        a->nbr = (ho_nbr*)realloc(a->nbr, sizeof(ho_nbr) * a->capNbr);
    }
    ho_nbr* n = &a->nbr[a->numNbr++];
    n->index = j;
    n->element = el;
    n->dr[0] = dr[0];
    n->dr[1] = dr[1];
    n->dr[2] = dr[2];
    n->d = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    n->dGdr = NULL;
}

/* Structure::calculateNeighborList (libnnp/Structure.cpp:287-399) */
static void ho_neighbor_list(int periodic, double const b[3][3], double rc)
{
    int pbc[3] = {0, 0, 0};
    if (periodic) ho_pbc_copies(b, rc, pbc);
    double const rc2 = rc * rc;
    for (int i = 0; i < g_n; ++i)
    {
        ho_atom* ai = &g_atoms[i];
        for (int j = 0; j < g_n; ++j)
        {
            for (int b0 = -pbc[0]; b0 <= pbc[0]; ++b0)
            for (int b1 = -pbc[1]; b1 <= pbc[1]; ++b1)
            for (int b2 = -pbc[2]; b2 <= pbc[2]; ++b2)
            {
                if (i == j && b0 == 0 && b1 == 0 && b2 == 0) continue;
                double dr[3];
                for (int k = 0; k < 3; ++k)
                {
                    dr[k] = ai->r[k] - g_atoms[j].r[k];
                    if (periodic)
                    {
                        dr[k] += b0 * b[0][k];
                        dr[k] += b1 * b[1][k];
                        dr[k] += b2 * b[2][k];
                    }
                }
                if (dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2] <= rc2)
                    ho_push_nbr(ai, j, g_atoms[j].element, dr);
            }
        }
    }
}

/* ---- symmetry functions (per-SF code path) ---------------------------- */

static double* ho_slot(ho_nbr* n, int slot) { return n->dGdr + 3 * slot; }

/* SymFncExpRad::calculate (libnnp/SymFncExpRad.cpp:119-180) */
static void ho_radial(ho_potential const* P, ho_atom* a, int s, ho_sf const* f)
{
    ho_cutoff const c = ho_make_cutoff(P->cutoffType, f->rc, P->cutoffAlpha);
    double result = 0.0;
    for (long j = 0; j < a->numNbr; ++j)
    {
        ho_nbr* n = &a->nbr[j];
        if (f->e1 != n->element || !(n->d < f->rc)) continue;
        double const rij = n->d;
        double pfc, pdfc;
        ho_fdf(&c, rij, &pfc, &pdfc);
        double const pexp = exp(-f->eta * (rij - f->rs) * (rij - f->rs));
        result += pexp * pfc;
        double const p1 = f->scalingFactor
                        * (pdfc - 2.0 * f->eta * (rij - f->rs) * pfc)
                        * pexp / rij;
        double* self = a->dGdrSelf + 3 * s;
        double* nb = ho_slot(n, f->slot[n->element]);
        for (int k = 0; k < 3; ++k)
        {
            self[k] += p1 * n->dr[k];
            nb[k] -= p1 * n->dr[k];
        }
    }
    a->G[s] = ho_scale(f, result);
}

/* SymFncExpAngn::calculate / SymFncExpAngw::calculate
 * (libnnp/SymFncExpAngn.cpp:83-222, SymFncExpAngw.cpp:83-205) */
static void ho_angular(ho_potential const* P, ho_atom* a, int s,
                       ho_sf const* f)
{
    int const narrow = (f->type == 3);
    ho_cutoff const c = ho_make_cutoff(P->cutoffType, f->rc, P->cutoffAlpha);
    double const pnorm = pow(2.0, 1.0 - f->zeta);
    double const pzl = f->zeta * f->lambda;
    double const rc2 = f->rc * f->rc;
    double result = 0.0;
    long const nn = a->numNbr ? a->numNbr : 1;
    for (long j = 0; j < nn - 1; ++j)
    {
        ho_nbr* nj = &a->nbr[j];
        int const nej = nj->element;
        double const rij = nj->d;
        if (!((f->e1 == nej || f->e2 == nej) && rij < f->rc)) continue;
        double const r2ij = rij * rij;
        double pfcij, pdfcij;
        ho_fdf(&c, rij, &pfcij, &pdfcij);
        for (long k = j + 1; k < a->numNbr; ++k)
        {
            ho_nbr* nk = &a->nbr[k];
            int const nek = nk->element;
            if (!((f->e1 == nej && f->e2 == nek)
                  || (f->e2 == nej && f->e1 == nek))) continue;
            double const rik = nk->d;
            if (!(rik < f->rc)) continue;
            double drjk[3] = {nk->dr[0] - nj->dr[0], nk->dr[1] - nj->dr[1],
                              nk->dr[2] - nj->dr[2]};
            double rjk = 0.0, pfcjk = 1.0, pdfcjk = 0.0;
            if (narrow)
            {
                rjk = drjk[0] * drjk[0] + drjk[1] * drjk[1]
                    + drjk[2] * drjk[2];
                if (!(rjk < rc2)) continue;
            }
            double pfcik, pdfcik;
            ho_fdf(&c, rik, &pfcik, &pdfcik);
            if (narrow)
            {
                rjk = sqrt(rjk);
                ho_fdf(&c, rjk, &pfcjk, &pdfcjk);
            }
            double costijk = nj->dr[0] * nk->dr[0] + nj->dr[1] * nk->dr[1]
                           + nj->dr[2] * nk->dr[2];
            double rinvijik = 1.0 / rij / rik;
            costijk *= rinvijik;
            double const pfc = narrow ? pfcij * pfcik * pfcjk : pfcij * pfcik;
            double const r2ik = rik * rik;
            double const rijs = rij - f->rs;
            double const riks = rik - f->rs;
            double const rjks = rjk - f->rs;
            double const pexp = narrow
                ? exp(-f->eta * (rijs * rijs + riks * riks + rjks * rjks))
                : exp(-f->eta * (rijs * rijs + riks * riks));
            double const plambda = 1.0 + f->lambda * costijk;
            double fg = pexp;
            if (plambda <= 0.0) fg = 0.0;
            else if (f->useIntegerPow) fg *= ho_pow_int(plambda, f->zetaInt - 1);
            else fg *= pow(plambda, f->zeta - 1.0);
            result += fg * plambda * pfc;
            fg *= pnorm;
            rinvijik *= pzl;
            costijk *= pzl;
            double const p2etapl = 2.0 * f->eta * plambda;
            double p1, p2, p3;
            if (narrow)
            {
                p1 = fg * (pfc * (rinvijik - costijk / r2ij - p2etapl * rijs
                           / rij) + pfcik * pfcjk * pdfcij * plambda / rij);
                p2 = fg * (pfc * (rinvijik - costijk / r2ik - p2etapl * riks
                           / rik) + pfcij * pfcjk * pdfcik * plambda / rik);
                p3 = fg * (pfc * (rinvijik + p2etapl * rjks / rjk) - pfcij
                           * pfcik * pdfcjk * plambda / rjk);
            }
            else
            {
                p1 = fg * (pfc * (rinvijik - costijk / r2ij - p2etapl * rijs
                           / rij) + pfcik * pdfcij * plambda / rij);
                p2 = fg * (pfc * (rinvijik - costijk / r2ik - p2etapl * riks
                           / rik) + pfcij * pdfcik * plambda / rik);
                p3 = fg * pfc * rinvijik;
            }
            double drij[3], drik[3];
            for (int q = 0; q < 3; ++q)
            {
                drij[q] = nj->dr[q] * (p1 * f->scalingFactor);
                drik[q] = nk->dr[q] * (p2 * f->scalingFactor);
                drjk[q] = drjk[q] * (p3 * f->scalingFactor);
            }
            double* self = a->dGdrSelf + 3 * s;
            double* sj = ho_slot(nj, f->slot[nej]);
            double* sk = ho_slot(nk, f->slot[nek]);
            for (int q = 0; q < 3; ++q)
            {
                self[q] += drij[q] + drik[q];
                sj[q] -= drij[q] + drjk[q];
                sk[q] -= drik[q] - drjk[q];
            }
        }
    }
    result *= pnorm;
    a->G[s] = ho_scale(f, result);
}

/* ---- NeuralNetwork (libnnp/NeuralNetwork.cpp:386-442, 761-896) -------- */

static void ho_activate(int af, double x, double* v, double* dv)
{
    double const lim = 35.0; /* EXP_LIMIT */
    switch (af)
    {
    case 0: *v = x; *dv = 1.0; return;
    case 1: { double const t = tanh(x); *v = t; *dv = 1.0 - t * t; return; }
    case 2:
        if (x > lim) { *v = 1.0; *dv = 0.0; return; }
        if (x < -lim) { *v = 0.0; *dv = 0.0; return; }
        { double const t = 1.0 / (1.0 + exp(-x)); *v = t; *dv = t * (1.0 - t); }
        return;
    case 3:
        if (x > lim) { *v = x; *dv = 1.0; return; }
        if (x < -lim) { *v = 0.0; *dv = 0.0; return; }
        { double t = exp(x); *v = log(1.0 + t); t = 1.0 / (1.0 + 1.0 / t); *dv = t; }
        return;
    case 4: if (x > 0.0) { *v = x; *dv = 1.0; } else { *v = 0.0; *dv = 0.0; }
        return;
    case 5: { double const t = exp(-0.5 * x * x); *v = t; *dv = -x * t; return; }
    case 6: *v = cos(x); *dv = -sin(x); return;
    case 7: { double const t = 1.0 / (1.0 + exp(-x)); *v = 1.0 - t;
              *dv = t * (t - 1.0); return; }
    case 8: { double const t = exp(-x); *v = t; *dv = -t; return; }
    default: *v = x * x; *dv = 2.0 * x; return;
    }
}

/* propagate + calculateDEdG (forward mode, as the reference). */
static void ho_network(ho_potential const* P, ho_atom* a)
{
    int const e = a->element;
    int const L = P->numLayers[e];
    int const* nn = P->neurons[e];
    double const* c = P->connections[e];
    int maxw = 0;
    for (int l = 0; l < L; ++l) if (nn[l] > maxw) maxw = nn[l];
    double* val = (double*)calloc((size_t)L * maxw, sizeof(double));
    double* dfdx = (double*)calloc((size_t)L * maxw, sizeof(double));
    long* woff = (long*)calloc((size_t)L, sizeof(long));
    long* boff = (long*)calloc((size_t)L, sizeof(long));
    long count = 0;
    for (int l = 1; l < L; ++l)
    {
        woff[l] = count;                 /* weight (in j, out k) at j*nout+k */
        count += (long)nn[l - 1] * nn[l];
        boff[l] = count;
        count += nn[l];
    }
    for (int k = 0; k < nn[0]; ++k) val[k] = a->G[k];
    for (int l = 1; l < L; ++l)
    {
        for (int i = 0; i < nn[l]; ++i)
        {
            double dtmp = 0.0;
            for (int j = 0; j < nn[l - 1]; ++j)
                dtmp += c[woff[l] + (long)j * nn[l] + i] * val[(l - 1) * maxw + j];
            dtmp += c[boff[l] + i];
            if (P->normalizeNeurons) dtmp /= nn[l - 1];
            ho_activate(P->activation[e][l], dtmp, &val[l * maxw + i],
                        &dfdx[l * maxw + i]);
        }
    }
    a->energy = val[(L - 1) * maxw + 0];
    int const H = L - 2;
    double* inner = (double*)calloc((size_t)maxw, sizeof(double));
    double* outer = (double*)calloc((size_t)maxw, sizeof(double));
    for (int k = 0; k < nn[0]; ++k)
    {
        for (int i = 0; i < nn[1]; ++i)
        {
            inner[i] = c[woff[1] + (long)k * nn[1] + i] * dfdx[1 * maxw + i];
            if (P->normalizeNeurons) inner[i] /= nn[0];
        }
        for (int l = 1; l < H + 1; ++l)
        {
            for (int i2 = 0; i2 < nn[l + 1]; ++i2)
            {
                outer[i2] = 0.0;
                for (int i1 = 0; i1 < nn[l]; ++i1)
                    outer[i2] += c[woff[l + 1] + (long)i1 * nn[l + 1] + i2]
                               * inner[i1];
                outer[i2] *= dfdx[(l + 1) * maxw + i2];
                if (P->normalizeNeurons) outer[i2] /= nn[l];
            }
            if (l < H)
                for (int i2 = 0; i2 < nn[l + 1]; ++i2) inner[i2] = outer[i2];
        }
        a->dEdG[k] = outer[0];
    }
    free(inner);
    free(outer);
    free(val);
    free(dfdx);
    free(woff);
    free(boff);
}

/* ---- prediction -------------------------------------------------------- */

int ho_predict(ho_potential const* P, int n, double const* box,
               double const* pos, int const* elem, double* energy,
               double* forces, double* atomic_energies)
{
    ho_constants();
    ho_free_atoms();
    if (n <= 0) return -1;
    g_n = n;
    g_atoms = (ho_atom*)calloc((size_t)n, sizeof(ho_atom));
    g_maxSF = 0;
    for (int e = 0; e < P->numElements; ++e)
        if (P->numSF[e] > g_maxSF) g_maxSF = P->numSF[e];
    double const L = P->normalize ? P->convLength : 1.0;
    double b[3][3] = {{0}}, inv[3][3] = {{0}};
    int const periodic = box != NULL;
    if (periodic)
    {
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) b[k][c] = box[3 * k + c];
        ho_inverse_box(b, inv);
    }
    for (int i = 0; i < n; ++i)
    {
        ho_atom* a = &g_atoms[i];
        a->element = elem[i];
        for (int k = 0; k < 3; ++k) a->r[k] = pos[3 * i + k];
        if (periodic) ho_remap(a->r, b, inv);
        /* Atom::toNormalizedUnits: r *= convLength */
        if (P->normalize) for (int k = 0; k < 3; ++k) a->r[k] *= L;
    }
    if (periodic && P->normalize)
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) b[k][c] *= L;
    double rcmax = 0.0;
    for (int e = 0; e < P->numElements; ++e)
        for (int s = 0; s < P->numSF[e]; ++s)
            if (P->sfs[e][s].rc > rcmax) rcmax = P->sfs[e][s].rc;
    ho_neighbor_list(periodic, b, rcmax);

    for (int i = 0; i < n; ++i)
    {
        ho_atom* a = &g_atoms[i];
        int const e = a->element;
        int const ns = P->numSF[e];
        a->numSF = ns;
        a->G = (double*)calloc((size_t)ns, sizeof(double));
        a->dEdG = (double*)calloc((size_t)ns, sizeof(double));
        a->dGdrSelf = (double*)calloc((size_t)ns * 3, sizeof(double));
        for (long k = 0; k < a->numNbr; ++k)
            a->nbr[k].dGdr = (double*)calloc(
                (size_t)(P->numSlots[e][a->nbr[k].element] + 1) * 3,
                sizeof(double));
        for (int s = 0; s < ns; ++s)
        {
            ho_sf const* f = &P->sfs[e][s];
            if (f->type == 2) ho_radial(P, a, s, f);
            else ho_angular(P, a, s, f);
        }
        ho_network(P, a);
    }

    /* Mode::calculateEnergy + Structure::toPhysicalUnits + addEnergyOffset */
    double E = 0.0;
    for (int i = 0; i < n; ++i) E += g_atoms[i].energy;
    if (P->normalize) E = E / P->convEnergy + n * P->meanEnergy;
    for (int e = 0; e < P->numElements; ++e)
    {
        long cnt = 0;
        for (int i = 0; i < n; ++i) cnt += (g_atoms[i].element == e);
        E += cnt * P->atomEnergy[e];
    }
    *energy = E;

    /* Mode::calculateForces (libnnp/Mode.cpp:1849-1912): self term plus,
     * for each unique neighbor j != i, the pair terms of j's entries that
     * point to i. */
    for (int i = 0; i < n; ++i)
    {
        ho_atom* ai = &g_atoms[i];
        double f[3] = {0.0, 0.0, 0.0};
        int const ei = ai->element;
        for (int s = 0; s < P->numSF[ei]; ++s)
            for (int q = 0; q < 3; ++q)
                f[q] -= ai->dEdG[s] * ai->dGdrSelf[3 * s + q];
        /* unique neighbors in ascending j (the list is j-major) */
        long last = -1;
        for (long k = 0; k < ai->numNbr; ++k)
        {
            long const j = ai->nbr[k].index;
            if (j == i || j == last) continue;
            last = j;
            ho_atom* aj = &g_atoms[j];
            int const ej = aj->element;
            for (long m = 0; m < aj->numNbr; ++m)
            {
                ho_nbr const* nb = &aj->nbr[m];
                if (nb->index != i) continue;
                int const ns = P->numSlots[ej][nb->element];
                /* table: SF index of slot t for neighbor element */
                for (int s = 0; s < P->numSF[ej]; ++s)
                {
                    int const t = P->sfs[ej][s].slot[nb->element];
                    if (t < 0 || t >= ns) continue;
                    for (int q = 0; q < 3; ++q)
                        f[q] -= aj->dEdG[s] * nb->dGdr[3 * t + q];
                }
            }
        }
        double const fs = P->normalize ? P->convEnergy / P->convLength : 1.0;
        for (int q = 0; q < 3; ++q)
        {
            forces[3 * i + q] = f[q] / fs;
            ai->f[q] = forces[3 * i + q];
        }
        if (atomic_energies)
            atomic_energies[i] = P->normalize ? ai->energy / P->convEnergy
                                              : ai->energy;
    }
    return 0;
}

void ho_cutoff_fdf(int type, double rc, double alpha, double r, double* fc,
                   double* dfc)
{
    ho_constants();
    ho_cutoff const c = ho_make_cutoff(type, rc, alpha);
    ho_fdf(&c, r, fc, dfc);
}

long ho_last_num_entries(void)
{
    long t = 0;
    for (int i = 0; i < g_n; ++i) t += g_atoms[i].numNbr;
    return t;
}

void ho_last_neighbors(long* counts, long* index, double* dr, double* d)
{
    long e = 0;
    for (int i = 0; i < g_n; ++i)
    {
        if (counts) counts[i] = g_atoms[i].numNbr;
        for (long k = 0; k < g_atoms[i].numNbr; ++k, ++e)
        {
            ho_nbr const* nb = &g_atoms[i].nbr[k];
            if (index) index[e] = nb->index;
            if (dr) for (int q = 0; q < 3; ++q) dr[3 * e + q] = nb->dr[q];
            if (d) d[e] = nb->d;
        }
    }
}

void ho_last_G(double* G, int stride)
{
    for (int i = 0; i < g_n; ++i)
    {
        ho_atom const* a = &g_atoms[i];
        for (int s = 0; s < stride; ++s)
            G[(long)i * stride + s] = (s < a->numSF) ? a->G[s] : 0.0;
    }
}
