/* Oracle: plain-C restatement of the reference's unstructured NS/SA path.
 * TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline); see
 * phx_oracle.h.  Line citations are to the reference project's files. */
#include "phx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OX_SMALL 1.0e-40   /* API/Common/include/Precision.h:27 */
#define OX_TINY 1.0e-40
#define OX_LARGE 1.0e40
#define OX_PI 3.141592653589793

static inline double omin(double a, double b) { return a < b ? a : b; }
static inline double omax(double a, double b) { return a > b ? a : b; }
static inline int ntot(const ox_grid *g) { return g->n_cell + g->n_bface; }

/* ------------------------------------------------------------------------ */
/* Metrics                                                                   */
/* ------------------------------------------------------------------------ */

/* UnstructGrid::ComputeFaceCenterAreaNormal3DNew2, Geo_UnstructGrid.cpp:5911-6043:
 * centre = node average, refined 4 times as the area-weighted centroid of the
 * fan triangles, then normal = sum of fan cross products. */
static void face_metrics(const ox_grid *g, ox_metrics *m)
{
    for (int f = 0; f < g->n_face; ++f) {
        int b = g->face_off[f], nn = g->face_off[f + 1] - b;
        double xc = 0, yc = 0, zc = 0;
        for (int j = 0; j < nn; ++j) {
            int p = g->face2node[b + j];
            xc += g->x[p]; yc += g->y[p]; zc += g->z[p];
        }
        double coef = 1.0 / nn;
        xc *= coef; yc *= coef; zc *= coef;
        double xn = 0, yn = 0, zn = 0;
        for (int cyc = 0; cyc < 5; ++cyc) {
            double xt = 0, yt = 0, zt = 0, at = 0;
            xn = yn = zn = 0;
            for (int j = 0; j < nn; ++j) {
                int p1 = g->face2node[b + j], p2 = g->face2node[b + (j + 1) % nn];
                double dx1 = g->x[p1] - xc, dy1 = g->y[p1] - yc, dz1 = g->z[p1] - zc;
                double dx2 = g->x[p2] - xc, dy2 = g->y[p2] - yc, dz2 = g->z[p2] - zc;
                double anx = dy1 * dz2 - dy2 * dz1;
                double any = dz1 * dx2 - dz2 * dx1;
                double anz = dx1 * dy2 - dx2 * dy1;
                double a = sqrt(anx * anx + any * any + anz * anz);
                double x00 = g->x[p1] + g->x[p2] + xc;
                double y00 = g->y[p1] + g->y[p2] + yc;
                double z00 = g->z[p1] + g->z[p2] + zc;
                at += a; xt += a * x00; yt += a * y00; zt += a * z00;
                xn += anx; yn += any; zn += anz;
            }
            if (at > OX_SMALL) {
                double t = 1.0 / at / 3.0;
                xc = xt * t; yc = yt * t; zc = zt * t;
            }
        }
        /* the fifth pass above is the final one of the reference: its normal
         * sums use the centre of the fourth refinement (computed before the
         * centre update of that same pass) */
        double a = sqrt(xn * xn + yn * yn + zn * zn);
        m->area[f] = a * 0.5;
        double oa = 1.0 / (a + OX_SMALL);
        m->xfn[f] = xn * oa; m->yfn[f] = yn * oa; m->zfn[f] = zn * oa;
        m->xfc[f] = xc; m->yfc[f] = yc; m->zfc[f] = zc;
    }
}

/* UnstructGrid::ComputeCellCenterVol3DNew2, Geo_UnstructGrid.cpp:6545-6819:
 * tetra decomposition (face centre, edge, cell node-average) for volume and
 * centroid; the centroid is kept only if it lies inside every face plane;
 * ghost centres mirror the owner across the face. */
static void cell_metrics(const ox_grid *g, ox_metrics *m)
{
    int nc = g->n_cell, nb = g->n_bface;
    double *xcc = m->xcc, *ycc = m->ycc, *zcc = m->zcc, *vol = m->vol;
    for (int c = 0; c < nc; ++c) {
        int b = g->cell_off[c], nn = g->cell_off[c + 1] - b;
        double xs = 0, ys = 0, zs = 0;
        for (int j = 0; j < nn; ++j) {
            int p = g->cell2node[b + j];
            xs += g->x[p]; ys += g->y[p]; zs += g->z[p];
        }
        xcc[c] = xs / nn; ycc[c] = ys / nn; zcc[c] = zs / nn;
    }
    double *xt = calloc(nc, sizeof(double)), *yt = calloc(nc, sizeof(double)), *zt = calloc(nc, sizeof(double));
    for (int c = 0; c < nc; ++c) vol[c] = 0.0;
    for (int f = 0; f < g->n_face; ++f) {
        int b = g->face_off[f], nn = g->face_off[f + 1] - b;
        int le = g->left[f], re = g->right[f];
        for (int j = 0; j < nn; ++j) {
            int p2 = g->face2node[b + j], p3 = g->face2node[b + (j + 1) % nn];
            double x21 = g->x[p2] - m->xfc[f], y21 = g->y[p2] - m->yfc[f], z21 = g->z[p2] - m->zfc[f];
            double x31 = g->x[p3] - m->xfc[f], y31 = g->y[p3] - m->yfc[f], z31 = g->z[p3] - m->zfc[f];
            double nx = y21 * z31 - y31 * z21;
            double ny = z21 * x31 - z31 * x21;
            double nz = x21 * y31 - x31 * y21;
            double x41 = xcc[le] - m->xfc[f], y41 = ycc[le] - m->yfc[f], z41 = zcc[le] - m->zfc[f];
            double xc = m->xfc[f] + g->x[p2] + g->x[p3] + xcc[le];
            double yc = m->yfc[f] + g->y[p2] + g->y[p3] + ycc[le];
            double zc = m->zfc[f] + g->z[p2] + g->z[p3] + zcc[le];
            double tmp = -(nx * x41 + ny * y41 + nz * z41);
            xt[le] += xc * tmp; yt[le] += yc * tmp; zt[le] += zc * tmp; vol[le] += tmp;
            if (f >= nb) {
                x41 = xcc[re] - m->xfc[f]; y41 = ycc[re] - m->yfc[f]; z41 = zcc[re] - m->zfc[f];
                xc = m->xfc[f] + g->x[p2] + g->x[p3] + xcc[re];
                yc = m->yfc[f] + g->y[p2] + g->y[p3] + ycc[re];
                zc = m->zfc[f] + g->z[p2] + g->z[p3] + zcc[re];
                tmp = nx * x41 + ny * y41 + nz * z41;
                xt[re] += xc * tmp; yt[re] += yc * tmp; zt[re] += zc * tmp; vol[re] += tmp;
            }
        }
    }
    for (int c = 0; c < nc; ++c) {
        double tmp = 1.0 / (4.0 * vol[c] + OX_SMALL);
        xt[c] *= tmp; yt[c] *= tmp; zt[c] *= tmp;
        vol[c] /= 6.0;
    }
    char *mark = malloc(nc);
    memset(mark, 1, nc);
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = g->right[f];
        double d = (xt[le] - m->xfc[f]) * m->xfn[f] + (yt[le] - m->yfc[f]) * m->yfn[f] + (zt[le] - m->zfc[f]) * m->zfn[f];
        if (d > 0.0) mark[le] = 0;
        if (f >= nb) {
            d = (xt[re] - m->xfc[f]) * m->xfn[f] + (yt[re] - m->yfc[f]) * m->yfn[f] + (zt[re] - m->zfc[f]) * m->zfn[f];
            if (d < 0.0) mark[re] = 0;
        }
    }
    for (int c = 0; c < nc; ++c)
        if (mark[c]) { xcc[c] = xt[c]; ycc[c] = yt[c]; zcc[c] = zt[c]; }
    free(mark); free(xt); free(yt); free(zt);
    for (int f = 0; f < nb; ++f) {
        int le = g->left[f], re = nc + f;
        if (m->area[f] > OX_SMALL) {
            double tmp = 2.0 * ((xcc[le] - m->xfc[f]) * m->xfn[f] + (ycc[le] - m->yfc[f]) * m->yfn[f] +
                                (zcc[le] - m->zfc[f]) * m->zfn[f]);
            xcc[re] = xcc[le] - m->xfn[f] * tmp;
            ycc[re] = ycc[le] - m->yfn[f] * tmp;
            zcc[re] = zcc[le] - m->zfn[f] * tmp;
        } else {
            xcc[re] = -xcc[le] + 2.0 * m->xfc[f];
            ycc[re] = -ycc[le] + 2.0 * m->yfc[f];
            zcc[re] = -zcc[le] + 2.0 * m->zfc[f];
        }
        vol[re] = vol[le];
    }
}

/* UnstructGrid::SkewnessSummary, Geo_UnstructGrid.cpp:2206-2330. */
static void skewness(const ox_grid *g, ox_metrics *m)
{
    int nc = g->n_cell, nb = g->n_bface;
    for (int c = 0; c < nc; ++c) m->skew[c] = 180.0;
    for (int f = nb; f < g->n_face; ++f) {
        if (m->area[f] <= OX_TINY) continue;
        int le = g->left[f], re = g->right[f];
        double x1 = m->xfc[f] - m->xcc[le], y1 = m->yfc[f] - m->ycc[le], z1 = m->zfc[f] - m->zcc[le];
        double d1 = sqrt(x1 * x1 + y1 * y1 + z1 * z1);
        double p1 = (m->xfn[f] * x1 + m->yfn[f] * y1 + m->zfn[f] * z1) / (d1 + OX_TINY);
        if (p1 > 1.0) p1 = 1.0;
        if (p1 < -1.0) p1 = -1.0;
        double x2 = m->xcc[re] - m->xfc[f], y2 = m->ycc[re] - m->yfc[f], z2 = m->zcc[re] - m->zfc[f];
        double d2 = sqrt(x2 * x2 + y2 * y2 + z2 * z2);
        double p2 = (m->xfn[f] * x2 + m->yfn[f] * y2 + m->zfn[f] * z2) / (d2 + OX_TINY);
        if (p2 > 1.0) p2 = 1.0;
        if (p2 < -1.0) p2 = -1.0;
        double ang = omin(asin(p1), asin(p2)) * 180.0 / OX_PI;
        m->skew[le] = omin(m->skew[le], ang);
        m->skew[re] = omin(m->skew[re], ang);
    }
    for (int f = 0; f < nb; ++f) {
        if (m->area[f] <= OX_TINY) continue;
        int le = g->left[f];
        double x1 = m->xfc[f] - m->xcc[le], y1 = m->yfc[f] - m->ycc[le], z1 = m->zfc[f] - m->zcc[le];
        double d1 = sqrt(x1 * x1 + y1 * y1 + z1 * z1);
        double p1 = (m->xfn[f] * x1 + m->yfn[f] * y1 + m->zfn[f] * z1) / (d1 + OX_TINY);
        if (p1 > 1.0) p1 = 1.0;
        if (p1 < -1.0) p1 = -1.0;
        m->skew[le] = omin(m->skew[le], asin(p1) * 180.0 / OX_PI);
    }
}

/* UnstructGrid::ComputeWeight, Geo_UnstructGrid.cpp:3761-3935 (3-D, every
 * face mark 1): per face the inverse squared centre distance, per cell the
 * inverse of sum_f w d d^T (zeroed when its determinant is below SMALL).
 * Boundary faces use the ghost centre. */
static void lsq_weights(const ox_grid *g, ox_metrics *m)
{
    int nc = g->n_cell, nb = g->n_bface;
    for (int c = 0; c < nc; ++c) m->ixx[c] = m->iyy[c] = m->izz[c] = m->ixy[c] = m->ixz[c] = m->iyz[c] = 0.0;
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double dx = (m->xcc[re] - m->xcc[le]) * 1.0;
        double dy = (m->ycc[re] - m->ycc[le]) * 1.0;
        double dz = (m->zcc[re] - m->zcc[le]) * 1.0;
        double ods = 1.0 / (dx * dx + dy * dy + dz * dz + OX_SMALL);
        double txx = ods * dx * dx, tyy = ods * dy * dy, tzz = ods * dz * dz;
        double txy = ods * dx * dy, txz = ods * dx * dz, tyz = ods * dy * dz;
        m->iwt[f] = ods;
        m->ixx[le] += txx; m->iyy[le] += tyy; m->izz[le] += tzz;
        m->ixy[le] += txy; m->ixz[le] += txz; m->iyz[le] += tyz;
        if (f >= nb) {
            m->ixx[re] += txx; m->iyy[re] += tyy; m->izz[re] += tzz;
            m->ixy[re] += txy; m->ixz[re] += txz; m->iyz[re] += tyz;
        }
    }
    for (int c = 0; c < nc; ++c) {
        double txx = m->ixx[c], tyy = m->iyy[c], tzz = m->izz[c];
        double txy = m->ixy[c], txz = m->ixz[c], tyz = m->iyz[c];
        double delt = (txx * tyy * tzz + 2.0 * txy * txz * tyz - txx * tyz * tyz - tyy * txz * txz - tzz * txy * txy);
        if (fabs(delt) < OX_SMALL) {
            m->ixx[c] = m->iyy[c] = m->izz[c] = m->ixy[c] = m->ixz[c] = m->iyz[c] = 0.0;
        } else {
            double od = 1.0 / delt;
            m->ixx[c] = (tyy * tzz - tyz * tyz) * od;
            m->iyy[c] = (txx * tzz - txz * txz) * od;
            m->izz[c] = (txx * tyy - txy * txy) * od;
            m->ixy[c] = (txz * tyz - txy * tzz) * od;
            m->ixz[c] = (txy * tyz - txz * tyy) * od;
            m->iyz[c] = (txy * txz - tyz * txx) * od;
        }
    }
}

void ox_lsq_weights(const ox_grid *g, ox_metrics *m) { lsq_weights(g, m); }

void ox_compute_metrics(const ox_grid *g, ox_metrics *m)
{
    face_metrics(g, m);
    cell_metrics(g, m);
    skewness(g, m);
    if (m->iwt) lsq_weights(g, m);
    double s = 0.0;
    for (int c = 0; c < g->n_cell; ++c) s += m->vol[c];
    m->avg_vol = s / (double)g->n_cell;
    /* UnstructGrid::ComputeCell2Face, Geo_UnstructGrid.cpp:1246-1290: faces in
     * ascending index order per cell. */
    if (m->c2f_off && m->c2f) {
        int nc = g->n_cell;
        int *cnt = calloc(nc + 1, sizeof(int));
        for (int f = 0; f < g->n_face; ++f) {
            cnt[g->left[f]]++;
            if (f >= g->n_bface) cnt[g->right[f]]++;
        }
        m->c2f_off[0] = 0;
        for (int c = 0; c < nc; ++c) m->c2f_off[c + 1] = m->c2f_off[c] + cnt[c];
        for (int c = 0; c < nc; ++c) cnt[c] = m->c2f_off[c];
        for (int f = 0; f < g->n_face; ++f) {
            m->c2f[cnt[g->left[f]]++] = f;
            if (f >= g->n_bface) m->c2f[cnt[g->right[f]]++] = f;
        }
        free(cnt);
    }
}

/* ------------------------------------------------------------------------ */
/* Boundary conditions (NSSolverUnstruct::Boundary, NSSolverUnstruct.cpp:13404-13515) */
/* ------------------------------------------------------------------------ */

/* SymmetryBCRegion, NSSolverUnstruct.cpp:19413-19455 (also inviscid walls). */
static void bc_symmetry(const ox_grid *g, const ox_metrics *m, int f, double *q, int nt)
{
    int le = g->left[f], re = g->n_cell + f;
    for (int k = 0; k < 5; ++k) q[k * nt + re] = q[k * nt + le];
    double uL = q[1 * nt + le], vL = q[2 * nt + le], wL = q[3 * nt + le];
    double vn = m->xfn[f] * uL + m->yfn[f] * vL + m->zfn[f] * wL;
    q[1 * nt + re] = uL - 2.0 * m->xfn[f] * vn;
    q[2 * nt + re] = vL - 2.0 * m->yfn[f] * vn;
    q[3 * nt + re] = wL - 2.0 * m->zfn[f] * vn;
}

/* ViscousAdiabaticWallBCRegion, NSSolverUnstruct.cpp:20988-21060 (no-slip,
 * static wall): ghost velocity is the reflection -u, density and pressure
 * copied. */
static void bc_adiabatic_wall(const ox_grid *g, int f, double *q, int nt)
{
    int le = g->left[f], re = g->n_cell + f;
    q[0 * nt + re] = q[0 * nt + le];
    q[1 * nt + re] = -q[1 * nt + le];
    q[2 * nt + re] = -q[2 * nt + le];
    q[3 * nt + re] = -q[3 * nt + le];
    q[4 * nt + re] = q[4 * nt + le];
}

/* FarfieldBCRegion, NSSolverUnstruct.cpp:21195-21330 (Riemann invariants). */
static void bc_farfield(const ox_grid *g, const ox_metrics *m, const ox_params *p, int f, double *q,
                        const double *gama, int nt)
{
    int le = g->left[f], re = g->n_cell + f;
    const double *pi = p->prim_inf;
    double rO = pi[0], uO = pi[1], vO = pi[2], wO = pi[3], pO = pi[4];
    double cO = sqrt(fabs(p->gama * pO / rO));
    double xn = m->xfn[f], yn = m->yfn[f], zn = m->zfn[f];
    for (int k = 0; k < 5; ++k) q[k * nt + re] = q[k * nt + le];
    double rI = q[le], uI = q[nt + le], vI = q[2 * nt + le], wI = q[3 * nt + le], pI = q[4 * nt + le];
    double vnO = xn * uO + yn * vO + zn * wO;
    double vnI = xn * uI + yn * vI + zn * wI;
    double gl = gama[le];
    double cI = sqrt(fabs(gl * pI / rI));
    double gm1 = gl - 1.0;
    double velI = sqrt(uI * uI + vI * vI + wI * wI);
    if (velI > cI) {
        if (vnI < 0.0)
            for (int k = 0; k < 5; ++k) q[k * nt + re] = pi[k];
        return;
    }
    double Rp = vnI + 2.0 * cI / gm1;
    double Rm = vnO - 2.0 * cO / gm1;
    double vnB = 0.5 * (Rp + Rm);
    double cB = 0.25 * (Rp - Rm) * gm1;
    double s, vtx, vty, vtz;
    if (vnB >= 0.0) {
        s = pI / pow(rI, gl);
        vtx = uI - xn * vnI; vty = vI - yn * vnI; vtz = wI - zn * vnI;
    } else {
        s = pO / pow(rO, gl);
        vtx = uO - xn * vnO; vty = vO - yn * vnO; vtz = wO - zn * vnO;
    }
    double rB = pow((cB * cB / (s * gl)), 1.0 / gm1);
    q[0 * nt + re] = rB;
    q[1 * nt + re] = vtx + xn * vnB;
    q[2 * nt + re] = vty + yn * vnB;
    q[3 * nt + re] = vtz + zn * vnB;
    q[4 * nt + re] = cB * cB * rB / gl;
}

static int is_wall(int t) { return t == OX_BC_SOLID_SURFACE; }

void ox_ns_boundary(const ox_grid *g, const ox_metrics *m, const ox_params *p, double *q, const double *gama)
{
    int nt = ntot(g);
    /* Regions are visited in region order; faces within a region in face order.
     * A face belongs to exactly one region, so visiting faces directly is
     * equivalent. */
    for (int f = 0; f < g->n_bface; ++f) {
        int t = g->region_type[g->bface_region[f]];
        if (is_wall(t)) {
            if (!p->viscous) bc_symmetry(g, m, f, q, nt);
            else bc_adiabatic_wall(g, f, q, nt);
        } else if (t == OX_BC_SYMMETRY) {
            bc_symmetry(g, m, f, q, nt);
        } else if (t == OX_BC_FARFIELD) {
            bc_farfield(g, m, p, f, q, gama, nt);
        } else if (t == OX_BC_INTERFACE) {
            /* NSSolverUnstruct::Boundary skips interface faces (:13474) */
        } else {
            /* extrapolation / outflow: ghost copies the owner */
            int le = g->left[f], re = g->n_cell + f;
            for (int k = 0; k < 5; ++k) q[k * nt + re] = q[k * nt + le];
        }
    }
}

/* NSSolverUnstruct::ComputeGamaAndTemperature, NSSolverUnstruct.cpp:4717-4730. */
void ox_gamma_temperature(const ox_grid *g, const ox_params *p, const double *q, double *gama, double *t)
{
    int nt = ntot(g);
    for (int c = 0; c < nt; ++c) {
        gama[c] = p->gama;
        t[c] = q[4 * nt + c] / (p->coef_state * q[c]);
    }
}

/* ------------------------------------------------------------------------ */
/* Gradient                                                                  */
/* ------------------------------------------------------------------------ */

/* UnstructGrid::CompGradientGGCell, Geo_UnstructGrid.cpp:3220-3284: ghost
 * gradients stay zero. */
static void gradient_ggcell(const ox_grid *g, const ox_metrics *m, const double *q, double *dx, double *dy,
                            double *dz)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    for (int c = 0; c < nt; ++c) dx[c] = dy[c] = dz[c] = 0.0;
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double qf = 0.5 * (q[le] + q[re]);
        double nx = m->xfn[f] * m->area[f], ny = m->yfn[f] * m->area[f], nz = m->zfn[f] * m->area[f];
        dx[le] += qf * nx; dy[le] += qf * ny; dz[le] += qf * nz;
        if (f >= nb) { dx[re] -= qf * nx; dy[re] -= qf * ny; dz[re] -= qf * nz; }
    }
    for (int c = 0; c < nc; ++c) {
        double ov = 1.0 / m->vol[c];
        dx[c] *= ov; dy[c] *= ov; dz[c] *= ov;
    }
}

/* UnstructGrid::CompGradientLSQ, Geo_UnstructGrid.cpp:3996-4085: weighted
 * differences to face neighbours (ghosts for boundary faces) times the
 * cell's inverse normal matrix; ghost gradients copy the owner's. */
static void gradient_lsq(const ox_grid *g, const ox_metrics *m, const double *q, double *dx, double *dy,
                         double *dz)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    for (int c = 0; c < nt; ++c) dx[c] = dy[c] = dz[c] = 0.0;
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double ddx = m->xcc[re] - m->xcc[le], ddy = m->ycc[re] - m->ycc[le], ddz = m->zcc[re] - m->zcc[le];
        double dq = m->iwt[f] * (q[re] - q[le]) * 1.0;
        double tx = dq * ddx, ty = dq * ddy, tz = dq * ddz;
        dx[le] += tx; dy[le] += ty; dz[le] += tz;
        if (f >= nb) { dx[re] += tx; dy[re] += ty; dz[re] += tz; }
    }
    for (int c = 0; c < nc; ++c) {
        double tx = dx[c], ty = dy[c], tz = dz[c];
        dx[c] = m->ixx[c] * tx + m->ixy[c] * ty + m->ixz[c] * tz;
        dy[c] = m->ixy[c] * tx + m->iyy[c] * ty + m->iyz[c] * tz;
        dz[c] = m->ixz[c] * tx + m->iyz[c] * ty + m->izz[c] * tz;
    }
    for (int f = 0; f < nb; ++f) {
        int le = g->left[f], re = nc + f;
        dx[re] = dx[le]; dy[re] = dy[le]; dz[re] = dz[le];
    }
}

void ox_gradient(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *f,
                 double *dfdx, double *dfdy, double *dfdz)
{
    if (p->gradient == 1) gradient_lsq(g, m, f, dfdx, dfdy, dfdz);
    else gradient_ggcell(g, m, f, dfdx, dfdy, dfdz);
}

/* ------------------------------------------------------------------------ */
/* Limiter                                                                   */
/* ------------------------------------------------------------------------ */

/* VenFun, API/Math/include/Math_Limiter.h:174-180. */
static inline double venfun(double x, double y, double eps)
{
    double x2 = x * x, xy = x * y, y2 = y * y;
    return (x2 + eps + 2.0 * xy) / (x2 + 2.0 * y2 + xy + eps);
}

/* Limiter::MinMaxDiff, Limiter.cpp:1202-1252 (boundary faces excluded, but
 * for interface faces). */
static void minmaxdiff(const ox_grid *g, const double *q, double *dmin, double *dmax)
{
    int nc = g->n_cell;
    for (int c = 0; c < nc; ++c) dmin[c] = dmax[c] = q[c];
    for (int f = 0; f < g->n_bface; ++f) {   /* interface ghosts count as neighbours (:1219-1231) */
        if (g->region_type[g->bface_region[f]] != OX_BC_INTERFACE) continue;
        int le = g->left[f];
        dmin[le] = omin(dmin[le], q[nc + f]); dmax[le] = omax(dmax[le], q[nc + f]);
    }
    for (int f = g->n_bface; f < g->n_face; ++f) {
        int le = g->left[f], re = g->right[f];
        dmin[le] = omin(dmin[le], q[re]); dmax[le] = omax(dmax[le], q[re]);
        dmin[re] = omin(dmin[re], q[le]); dmax[re] = omax(dmax[re], q[le]);
    }
    for (int c = 0; c < nc; ++c) { dmin[c] -= q[c]; dmax[c] -= q[c]; }
}

/* Limiter::VencatLimiter7, Limiter.cpp:1091-1200 (3-D: n = 3). */
static void vencat7(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                    const double *dqdx, const double *dqdy, const double *dqdz, double *limit)
{
    int nc = g->n_cell, nb = g->n_bface;
    double *dmin = malloc(sizeof(double) * nc), *dmax = malloc(sizeof(double) * nc);
    double *eps = malloc(sizeof(double) * nc);
    minmaxdiff(g, q, dmin, dmax);
    double K = p->venkat_coeff;
    double eps_tmp = K * K * K;
    eps_tmp *= 1.0 / pow(pow(m->avg_vol, 1.0 / 3.0), 3.0);
    for (int c = 0; c < nc; ++c) {
        eps[c] = eps_tmp * q[c] * q[c];
        eps[c] *= pow(pow(m->vol[c], 1.0 / 3.0), 3.0);
    }
    for (int f = 0; f < g->n_face; ++f) {
        for (int side = 0; side < (f < nb ? 1 : 2); ++side) {
            int c = side == 0 ? g->left[f] : g->right[f];
            double dx = m->xfc[f] - m->xcc[c], dy = m->yfc[f] - m->ycc[c], dz = m->zfc[f] - m->zcc[c];
            double dqf = dqdx[c] * dx + dqdy[c] * dy + dqdz[c] * dz;
            if (dqf > OX_SMALL) limit[c] = omin(limit[c], venfun(dmax[c], dqf, eps[c]));
            else if (dqf < -OX_SMALL) limit[c] = omin(limit[c], venfun(dmin[c], dqf, eps[c]));
        }
    }
    free(dmin); free(dmax); free(eps);
}

/* NSSolverUnstruct::ComputeLimiter (NSSolverUnstruct.cpp:18189-18240) with a
 * scalar Venkatakrishnan limiter from rho and p (limitVariables=0,
 * limitVector=0, Limiter.cpp:91-135), then SetLimitBoundary
 * (Geo_UnstructGrid.cpp:10744-10775): zero on both sides of far-field /
 * inflow faces.  `limit` holds nTotal values. */
/* Limiter::BarthLimiter, API/Physics/src/Limiter.cpp:157-262: for each cell
 * and each of its faces (boundary faces from the owner only), the face
 * extrapolation dq = grad . (x_f - x_c) is limited to the neighbour min/max
 * differences; a face whose centre lies behind the cell's outward normal
 * zeroes the limiter. */
static void barth_face(int c, double xn, double yn, double zn, double sgn, const ox_metrics *m, int f,
                       const double *dqdx, const double *dqdy, const double *dqdz, const double *dmin,
                       const double *dmax, double *limit)
{
    double dx = m->xfc[f] - m->xcc[c], dy = m->yfc[f] - m->ycc[c], dz = m->zfc[f] - m->zcc[c];
    double dq = dqdx[c] * dx + dqdy[c] * dy + dqdz[c] * dz;
    double ds = sqrt(dx * dx + dy * dy + dz * dz);
    double dot = sgn * (xn * dx + yn * dy + zn * dz) / (ds + OX_SMALL);
    if (dot < 0.0) limit[c] = 0.0;
    else if (dq > dmax[c]) limit[c] = omin(limit[c], dmax[c] / (dq + OX_SMALL));
    else if (dq < dmin[c]) limit[c] = omin(limit[c], dmin[c] / (dq + OX_SMALL));
}

static void barth(const ox_grid *g, const ox_metrics *m, const double *q, const double *dqdx, const double *dqdy,
                  const double *dqdz, double *limit)
{
    int nc = g->n_cell, nb = g->n_bface;
    double *dmin = malloc(sizeof(double) * (size_t)nc), *dmax = malloc(sizeof(double) * (size_t)nc);
    minmaxdiff(g, q, dmin, dmax);
    for (int f = 0; f < g->n_face; ++f) {
        barth_face(g->left[f], m->xfn[f], m->yfn[f], m->zfn[f], 1.0, m, f, dqdx, dqdy, dqdz, dmin, dmax, limit);
        if (f >= nb)
            barth_face(g->right[f], m->xfn[f], m->yfn[f], m->zfn[f], -1.0, m, f, dqdx, dqdy, dqdz, dmin, dmax,
                       limit);
    }
    free(dmin);
    free(dmax);
}

void ox_limiter(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                const double *dqdx, const double *dqdy, const double *dqdz, double *limit)
{
    int nt = ntot(g);
    for (int c = 0; c < nt; ++c) limit[c] = 1.0;
    if (p->limiter == OX_LIMITER_NOLIM) return;
    if (p->first_order) {   /* NSSolverUnstruct::ComputeLimiter :18215-18224: zero, no limiter */
        for (int c = 0; c < nt; ++c) limit[c] = 0.0;
        return;
    }
    if (p->limiter == OX_LIMITER_BARTH) {
        barth(g, m, q, dqdx, dqdy, dqdz, limit);
        barth(g, m, q + 4 * nt, dqdx + 4 * nt, dqdy + 4 * nt, dqdz + 4 * nt, limit);
    } else {
        vencat7(g, m, p, q, dqdx, dqdy, dqdz, limit);
        vencat7(g, m, p, q + 4 * nt, dqdx + 4 * nt, dqdy + 4 * nt, dqdz + 4 * nt, limit);
    }
    for (int f = 0; f < g->n_bface; ++f) {
        int t = g->region_type[g->bface_region[f]];
        if (t != OX_BC_INTERFACE && t != OX_BC_SYMMETRY && !is_wall(t) && t != OX_BC_OUTFLOW) {
            limit[g->left[f]] = 0.0;
            limit[g->n_cell + f] = 0.0;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Inviscid flux                                                             */
/* ------------------------------------------------------------------------ */

/* Harten fix, API/Physics/include/Flux_RoeEntropyCorrection.h:66-74. */
static inline double harten(double e, double lim)
{
    double a = fabs(e);
    if (a < lim) a = 0.5 * (e * e + lim * lim) / lim;
    return a;
}

/* Roe_Scheme_ConservativeForm, API/Physics/src/Flux_Inviscid.cpp:136-399
 * (perfect gas, no preconditioning, static grid), with the entropy fix of
 * Flux_RoeEntropyCorrection method 3 (Flux_RoeEntropyCorrection.cpp:126-135).
 * Returns the flux per unit area in f[5]. */
static void roe_flux(const double *ql, const double *qr, double gl, double gr, double xsn, double ysn,
                     double zsn, double acoustic, double convective, double *f)
{
    const double LITTLE = 1.0e-10;
    double rL = omax(ql[0], LITTLE), uL = ql[1], vL = ql[2], wL = ql[3], pL = omax(ql[4], LITTLE);
    double rR = omax(qr[0], LITTLE), uR = qr[1], vR = qr[2], wR = qr[3], pR = omax(qr[4], LITTLE);
    double v2L = uL * uL + vL * vL + wL * wL;
    double v2R = uR * uR + vR * vR + wR * wR;
    double hL = (gl / (gl - 1.0)) * (pL / rL) + 0.5 * v2L;
    double hR = (gr / (gr - 1.0)) * (pR / rR) + 0.5 * v2R;
    double vnL = xsn * uL + ysn * vL + zsn * wL;
    double vnR = xsn * uR + ysn * vR + zsn * wR;
    double rvnL = rL * vnL, rvnR = rR * vnR;
    f[0] = 0.5 * (rvnL + rvnR);
    f[1] = 0.5 * (rvnL * uL + xsn * pL + rvnR * uR + xsn * pR);
    f[2] = 0.5 * (rvnL * vL + ysn * pL + rvnR * vR + ysn * pR);
    f[3] = 0.5 * (rvnL * wL + zsn * pL + rvnR * wR + zsn * pR);
    f[4] = 0.5 * (rvnL * hL + rvnR * hR);
    double ratio = sqrt(rR / rL);
    double coef = 1.0 / (1.0 + ratio);
    double um = (uL + uR * ratio) * coef;
    double vm = (vL + vR * ratio) * coef;
    double wm = (wL + wR * ratio) * coef;
    double pm = (pL + pR * ratio) * coef;
    double rm = sqrt(rL * rR);
    double gama = (gl + gr * ratio) * coef;
    double gm1 = gama - 1.0;
    double v2 = um * um + vm * vm + wm * wm;
    double absv = sqrt(v2);
    double hm = gama / gm1 * pm / rm + 0.5 * v2;
    double vn = xsn * um + ysn * vm + zsn * wm;
    double theta = vn;
    double c2 = gm1 * (hm - 0.5 * v2);
    double cm = sqrt(fabs(c2));
    double e1 = fabs(vn), e2 = fabs(vn + cm), e3 = fabs(vn - cm);
    (void)absv;
    double EL = (1.0 / (gl - 1.0)) * (pL / rL) + 0.5 * v2L;
    double ER = (1.0 / (gr - 1.0)) * (pR / rR) + 0.5 * v2R;
    double dq0 = rR - rL, dq1 = rR * uR - rL * uL, dq2 = rR * vR - rL * vL, dq3 = rR * wR - rL * wL;
    double dq4 = rR * ER - rL * EL;
    double maxe = fabs(vn) + cm;
    e1 = harten(e1, convective * maxe);
    e2 = harten(e2, acoustic * maxe);
    e3 = harten(e3, acoustic * maxe);
    double xi1 = (2.0 * e1 - e2 - e3) / (2.0 * c2);
    double xi2 = (e2 - e3) / (2.0 * cm);
    double dc = theta * dq0 - xsn * dq1 - ysn * dq2 - zsn * dq3;
    double c2dc = c2 * dc;
    double dh = -gm1 * (um * dq1 + vm * dq2 + wm * dq3 - dq4) + 0.5 * gm1 * v2 * dq0;
    f[0] -= 0.5 * (e1 * dq0 - dh * xi1 - dc * xi2);
    f[1] -= 0.5 * (e1 * dq1 + (xsn * c2dc - um * dh) * xi1 + (xsn * dh - um * dc) * xi2);
    f[2] -= 0.5 * (e1 * dq2 + (ysn * c2dc - vm * dh) * xi1 + (ysn * dh - vm * dc) * xi2);
    f[3] -= 0.5 * (e1 * dq3 + (zsn * c2dc - wm * dh) * xi1 + (zsn * dh - wm * dc) * xi2);
    f[4] -= 0.5 * (e1 * dq4 + (theta * c2dc - hm * dh) * xi1 + (theta * dh - hm * dc) * xi2);
}

/* The other schemes of GetINVScheme (API/Physics/src/Flux_Inviscid.cpp:88-134)
 * for a perfect gas on a static grid (face velocity 0), without
 * preconditioning; each returns the flux per unit area in f[5]. */
#define OX_SMALL 1.0e-40

/* Steger_Scheme, Flux_Inviscid.cpp:12467-12694, entropy fix method 3 (none):
 * positive eigenvalues of the left state plus negative ones of the right. */
static void steger_side(const double *q, double g, double xsn, double ysn, double zsn, double sgn, double *f)
{
    double r = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
    double v2 = u * u + v * v + w * w;
    double h = (g / (g - 1.0)) * (p / r) + 0.5 * v2;
    double e = h - p / (r + OX_SMALL);
    double vn = xsn * u + ysn * v + zsn * w;
    double c2 = g * p / r;
    double c = sqrt(fabs(c2));
    double l1 = vn, l2 = vn + c, l3 = vn - c;
    l1 = 0.5 * (l1 + sgn * fabs(l1));
    l2 = 0.5 * (l2 + sgn * fabs(l2));
    l3 = 0.5 * (l3 + sgn * fabs(l3));
    double c2g = c2 / g;
    double xi1 = c2g * (l1 + l1 - l2 - l3) / (c2 + c2);
    double xi2 = c2g * (l2 - l3) / (c + c);
    double ex = l1 - xi1;
    f[0] = r * ex;
    f[1] = r * (ex * u + xi2 * xsn);
    f[2] = r * (ex * v + xi2 * ysn);
    f[3] = r * (ex * w + xi2 * zsn);
    f[4] = r * (l1 * e - xi1 * h + xi2 * vn);
}

static void steger_flux(const double *ql, const double *qr, double gl, double gr, double xsn, double ysn,
                        double zsn, double *f)
{
    double a[5], b[5];
    steger_side(ql, gl, xsn, ysn, zsn, 1.0, a);
    steger_side(qr, gr, xsn, ysn, zsn, -1.0, b);
    for (int k = 0; k < 5; ++k) f[k] = a[k] + b[k];
}

/* Vanleer_Scheme, Flux_Inviscid.cpp:12697-12950 (nPrecondition = 0):
 * Van Leer's Mach-number splitting, F+ of the left state plus F- of the right. */
static void vanleer_side(const double *q, double g, double xsn, double ysn, double zsn, int left, double *f)
{
    double r = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
    double v2 = u * u + v * v + w * w;
    double h = (g / (g - 1.0)) * (p / r) + 0.5 * v2;
    double vn = xsn * u + ysn * v + zsn * w;
    double rvn = r * vn;
    double c = sqrt(fabs(g * p / r));
    double mach = vn / c;
    int full = left ? mach > 1.0 : mach < -1.0;
    int none = left ? mach < -1.0 : mach > 1.0;
    if (full) {
        f[0] = rvn;
        f[1] = rvn * u + xsn * p;
        f[2] = rvn * v + ysn * p;
        f[3] = rvn * w + zsn * p;
        f[4] = rvn * h;
    } else if (none) {
        for (int k = 0; k < 5; ++k) f[k] = 0.0;
    } else {
        double fm, t;
        if (left) {
            fm = 0.25 * r * c * (mach + 1.0) * (mach + 1.0);
            t = (-vn + 2.0 * c) / g;
        } else {
            fm = -0.25 * r * c * (mach - 1.0) * (mach - 1.0);
            t = (-vn - 2.0 * c) / g;
        }
        f[0] = fm;
        f[1] = fm * (u + xsn * t);
        f[2] = fm * (v + ysn * t);
        f[3] = fm * (w + zsn * t);
        f[4] = fm * h;
    }
}

static void vanleer_flux(const double *ql, const double *qr, double gl, double gr, double xsn, double ysn,
                         double zsn, double *f)
{
    double a[5], b[5];
    vanleer_side(ql, gl, xsn, ysn, zsn, 1, a);
    vanleer_side(qr, gr, xsn, ysn, zsn, 0, b);
    for (int k = 0; k < 5; ++k) f[k] = a[k] + b[k];
}

/* GetAngleOfTwoVector (API/DataStruct/include/PHMatrix.h:203-217): the dot
 * product over both norms (DotProduct, GetNorm: sums from zero), clamped, acos. */
static double angle_of(const double *a, const double *b)
{
    double dot = 0.0, na = 0.0, nb = 0.0;
    for (int i = 0; i < 3; ++i) dot += a[i] * b[i];
    for (int i = 0; i < 3; ++i) na += a[i] * a[i];
    for (int i = 0; i < 3; ++i) nb += b[i] * b[i];
    double c = dot / sqrt(na) / sqrt(nb);
    if (c > 1.0) return 0.0;
    if (c < -1.0) return OX_PI;
    return acos(c);
}

/* CrossProduct (API/Math/src/Math_BasisFunction.cpp:98-104). */
static void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

/* Rotate_Vanleer_Scheme (Flux_Inviscid.cpp:12952-13180): Van Leer's splitting
 * along n1, the direction of the velocity jump across the face (x when there
 * is none), turned to the face normal's side, and along n2, normal to n1 in
 * the plane of n1 and the face normal (y when n1 is the normal), each weighted
 * by the cosine of its angle to the face normal. */
static void vanleer_rotate_flux(const double *ql, const double *qr, double gl, double gr, double xsn, double ysn,
                                double zsn, double *f)
{
    const double n[3] = {xsn, ysn, zsn};
    double n1[3], n2[3];
    const double du = qr[1] - ql[1], dv = qr[2] - ql[2], dw = qr[3] - ql[3];
    if (du == 0 && dv == 0 && dw == 0) {
        n1[0] = 1; n1[1] = 0; n1[2] = 0;
    } else {
        const double sqdv = sqrt(pow(du, 2) + pow(dv, 2) + pow(dw, 2));
        n1[0] = du / sqdv; n1[1] = dv / sqdv; n1[2] = dw / sqdv;
    }
    double angle1 = angle_of(n1, n);
    if (cos(angle1) < 0) {
        n1[0] = -n1[0]; n1[1] = -n1[1]; n1[2] = -n1[2];
        angle1 = angle_of(n1, n);
    }
    if (fabs(n1[0] - xsn) < 1.0e-8 && fabs(n1[1] - ysn) < 1.0e-8 && fabs(n1[2] - zsn) < 1.0e-8) {
        n2[0] = 0; n2[1] = 1; n2[2] = 0;
    } else {
        double t[3];
        cross3(n1, n, t);
        cross3(t, n1, n2);
    }
    double nn = 0.0;
    for (int i = 0; i < 3; ++i) nn += n2[i] * n2[i];
    const double normn2 = sqrt(nn);
    if (cos(angle_of(n2, n)) < 0) {
        n2[0] = -n2[0] / normn2; n2[1] = -n2[1] / normn2; n2[2] = -n2[2] / normn2;
    } else {
        n2[0] = n2[0] / normn2; n2[1] = n2[1] / normn2; n2[2] = n2[2] / normn2;
    }
    const double angle2 = angle_of(n2, n);
    for (int k = 0; k < 5; ++k) f[k] = 0.0;
    for (int dir = 1; dir <= 2; ++dir) {
        const double *d = dir == 1 ? n1 : n2;
        double a[5], b[5];
        vanleer_side(ql, gl, d[0], d[1], d[2], 1, a);
        vanleer_side(qr, gr, d[0], d[1], d[2], 0, b);
        const double c = cos(dir == 1 ? angle1 : angle2);
        for (int k = 0; k < 5; ++k) f[k] = f[k] + c * (a[k] + b[k]);
    }
}

/* Hlle_Scheme, Flux_Inviscid.cpp:13917-14077: the HLLE flux with signal
 * speeds from the Roe average and both sides; the conserved jump from
 * PerfectGas::Primitive2Conservative (PerfectGas.cpp:284-323). */
static void hlle_flux(const double *ql, const double *qr, double gl, double gr, double xsn, double ysn,
                      double zsn, double *f)
{
    double rl = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
    double rr = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
    double v2l = ul * ul + vl * vl + wl * wl;
    double v2r = ur * ur + vr * vr + wr * wr;
    double hl = (gl / (gl - 1.0)) * (pl / rl) + 0.5 * v2l;
    double hr = (gr / (gr - 1.0)) * (pr / rr) + 0.5 * v2r;
    double ratio = sqrt(rr / rl);
    double coef = 1.0 / (1.0 + ratio);
    double rm = sqrt(rl * rr);
    double um = (ul + ur * ratio) * coef;
    double vm = (vl + vr * ratio) * coef;
    double wm = (wl + wr * ratio) * coef;
    double pm = (pl + pr * ratio) * coef;
    double gm = (gl + gr * ratio) * coef;
    double vnl = xsn * ul + ysn * vl + zsn * wl;
    double vnr = xsn * ur + ysn * vr + zsn * wr;
    double rvnl = rl * vnl, rvnr = rr * vnr;
    double vn = xsn * um + ysn * vm + zsn * wm;
    double cl = sqrt(gl * pl / (rl + OX_SMALL));
    double cr = sqrt(gr * pr / (rr + OX_SMALL));
    double cm = sqrt(gm * pm / (rm + OX_SMALL));
    double fl[5] = {rvnl, rvnl * ul + xsn * pl, rvnl * vl + ysn * pl, rvnl * wl + zsn * pl, rvnl * hl};
    double fr[5] = {rvnr, rvnr * ur + xsn * pr, rvnr * vr + ysn * pr, rvnr * wr + zsn * pr, rvnr * hr};
    double el = (pl / rl) / (gl - 1.0) + 0.5 * v2l;
    double er = (pr / rr) / (gr - 1.0) + 0.5 * v2r;
    double ul5[5] = {rl, rl * ul, rl * vl, rl * wl, rl * el};
    double ur5[5] = {rr, rr * ur, rr * vr, rr * wr, rr * er};
    double bm = omin(0.0, omin(vn - cm, vnl - cl));
    double bp = omax(0.0, omax(vn + cm, vnr + cr));
    double c1 = bp * bm / (bp - bm + OX_SMALL);
    double c2 = -0.5 * (bp + bm) / (bp - bm + OX_SMALL);
    for (int k = 0; k < 5; ++k) f[k] = 0.5 * (fl[k] + fr[k]) + c1 * (ur5[k] - ul5[k]) + c2 * (fr[k] - fl[k]);
}

/* Ausmdv_Scheme, Flux_Inviscid.cpp:13191-13461: AUSMD / AUSMV blended by the
 * pressure jump, the Haenel / Van Leer flux at shocks, and its entropy fix. */
static void ausmdv_flux(const double *ql, const double *qr, double gl, double gr, double xsn, double ysn,
                        double zsn, double *f)
{
    double rl = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
    double rr = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
    double gama = 0.5 * (gl + gr);
    double v2l = ul * ul + vl * vl + wl * wl;
    double v2r = ur * ur + vr * vr + wr * wr;
    double hl = (gl / (gl - 1.0)) * (pl / rl) + 0.5 * v2l;
    double hr = (gr / (gr - 1.0)) * (pr / rr) + 0.5 * v2r;
    double vnl = xsn * ul + ysn * vl + zsn * wl;
    double vnr = xsn * ur + ysn * vr + zsn * wr;
    double orl = 1.0 / (rl + OX_SMALL), orr = 1.0 / (rr + OX_SMALL);
    double cl = sqrt(gama * pl * orl), cr = sqrt(gama * pr * orr);
    double cm = omax(cl, cr);
    double ocm = 1.0 / (cm + OX_SMALL);
    double ssw = ((vnl > cl && vnr < cr) || (vnl > -cl && vnr < -cr)) ? 1.0 : 0.0;
    double ssw_a = 1.0 - ssw;
    /* Haenel / Van Leer with the side sound speeds */
    double ml = vnl / cl, mr = vnr / cr;
    double mla = fabs(ml), mra = fabs(mr);
    double mpl, ppl, mmr, pmr;
    if (mla >= 1.0) { mpl = 0.5 * (ml + mla); ppl = 0.5 * (1.0 + ml / (mla + OX_SMALL)); }
    else { double t = 0.25 * ((ml + 1.0) * (ml + 1.0)); mpl = t; ppl = t * (2.0 - ml); }
    if (mra >= 1.0) { mmr = 0.5 * (mr - mra); pmr = 0.5 * (1.0 - mr / (mra + OX_SMALL)); }
    else { double t = 0.25 * ((mr - 1.0) * (mr - 1.0)); mmr = -t; pmr = t * (2.0 + mr); }
    double p12 = ppl * pl + pmr * pr;
    double rvnl_v = cl * rl * mpl, rvnr_v = cr * rr * mmr;
    /* AUSMD / AUSMV with the common sound speed */
    ml = vnl * ocm; mla = fabs(ml);
    mr = vnr * ocm; mra = fabs(mr);
    double r1 = pl * orl, r2 = pr * orr, r3 = 2.0 / (r1 + r2);
    double al = r1 * r3, ar = r2 * r3;
    if (mla >= 1.0) mpl = 0.5 * (ml + mla);
    else { double t = 0.25 * ((ml + 1.0) * (ml + 1.0)); mpl = al * t + (1.0 - al) * (0.5 * (ml + mla)); }
    if (mra >= 1.0) mmr = 0.5 * (mr - mra);
    else { double t = 0.25 * ((mr - 1.0) * (mr - 1.0)); mmr = -ar * t + (1.0 - ar) * (0.5 * (mr - mra)); }
    double rvnl_d = cm * rl * mpl, rvnr_d = cm * rr * mmr;
    double rvn = rvnl_d + rvnr_d;
    rvnl_d = 0.5 * (rvn + fabs(rvn));
    rvnr_d = 0.5 * (rvn - fabs(rvn));
    double rvnl = rvnl_v, rvnr = rvnr_v;
    double s = 0.5 * omin(1.0, 10.0 * fabs(pr - pl) / omin(pl, pr));
    double rvvn = ssw * (rvnl_v * vnl + rvnr_v * vnr);
    rvvn += (0.5 - s) * ssw_a * (rvnl_d * vnl + rvnr_d * vnr) + (0.5 + s) * ssw_a * cm * (rl * mpl * vnl + rr * mmr * vnr);
    int a = (vnl - cl) < 0.0 && (vnr - cr) > 0.0;
    int b = (vnl + cl) < 0.0 && (vnr + cr) > 0.0;
    if (a && !b) {
        double t = ssw_a * 0.125 * ((vnr - cr) - (vnl - cl));
        rvnl += t * rl; rvnr -= t * rr;
    } else if (!a && b) {
        double t = ssw_a * 0.125 * ((vnr + cr) - (vnl + cl));
        rvnl += t * rl; rvnr -= t * rr;
    }
    double dul = ul - xsn * vnl, dvl = vl - ysn * vnl, dwl = wl - zsn * vnl;
    double dur = ur - xsn * vnr, dvr = vr - ysn * vnr, dwr = wr - zsn * vnr;
    rvvn += p12;
    f[0] = rvnl + rvnr;
    f[1] = rvnl * dul + rvnr * dur + rvvn * xsn;
    f[2] = rvnl * dvl + rvnr * dvr + rvvn * ysn;
    f[3] = rvnl * dwl + rvnr * dwr + rvvn * zsn;
    f[4] = rvnl * hl + rvnr * hr;
}

/* FMmpn / FMppn, Flux_Inviscid.cpp:14079-14107: split Mach number and
 * pressure polynomials (ipn = +1 for the left side, -1 for the right). */
static double fm_mpn(double m, double ipn)
{
    if (fabs(m) >= 1.0) return 0.5 * (m + ipn * fabs(m));
    return ipn * 0.25 * ((m + ipn) * (m + ipn));
}

static double fm_ppn(double m, double ipn)
{
    if (fabs(m) >= 1.0) return 0.5 * (m + ipn * fabs(m)) / m;
    return ipn * 0.25 * ((m + ipn) * (m + ipn)) * (2.0 * ipn - m);
}

/* AusmpwPlus_Scheme, Flux_Inviscid.cpp:13628-13915: AUSMPW+ with the mean
 * sound speed 0.5 (a_L + a_R) and the pressure-ratio weight
 * 1 - min(p_L/p_R, p_R/p_L)^3 * AusmpwPlusLimiter. */
static void ausmpwp_flux(const double *ql, const double *qr, double gl, double gr, double xsn, double ysn,
                         double zsn, double lim, double *f)
{
    double rl = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
    double rr = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
    double v2l = ul * ul + vl * vl + wl * wl;
    double v2r = ur * ur + vr * vr + wr * wr;
    double hl = (gl / (gl - 1.0)) * (pl / rl) + 0.5 * v2l;
    double hr = (gr / (gr - 1.0)) * (pr / rr) + 0.5 * v2r;
    double al = sqrt(gl * (pl / (rl + OX_SMALL)));
    double ar = sqrt(gr * (pr / (rr + OX_SMALL)));
    double vnl = xsn * ul + ysn * vl + zsn * wl;
    double vnr = xsn * ur + ysn * vr + zsn * wr;
    double minplr = omin(pl / (pr + OX_SMALL), pr / (pl + OX_SMALL));
    double c12 = 0.5 * (al + ar);
    double ocm = 1.0 / c12;
    double ml = vnl * ocm, mr = vnr * ocm;
    double fm4l = fm_mpn(ml, 1.0), fm4r = fm_mpn(mr, -1.0);
    double fp5l = fm_ppn(ml, 1.0), fp5r = fm_ppn(mr, -1.0);
    double m12 = fm4l + fm4r;
    double p12 = fp5l * pl + fp5r * pr;
    double fw = 1.0 - minplr * minplr * minplr * lim;
    double op12 = 1.0 / (p12 + OX_SMALL);
    double fl = 0.0, fr = 0.0;
    if (p12 != 0.0) {
        if (fabs(ml) <= 1.0) fl = pl * op12 - 1.0;
        if (fabs(mr) <= 1.0) fr = pr * op12 - 1.0;
    }
    double mpl, mmr;
    if (m12 >= 0.0) {
        double o = 1.0 + fr;
        mpl = fm4l + fm4r * ((1.0 - fw) * o - fl);
        mmr = fm4r * fw * o;
    } else {
        double o = 1.0 + fl;
        mpl = fm4l * fw * o;
        mmr = fm4r + fm4l * ((1.0 - fw) * o - fr);
    }
    f[0] = c12 * (mpl * rl + mmr * rr);
    f[1] = c12 * (mpl * rl * ul + mmr * rr * ur) + p12 * xsn;
    f[2] = c12 * (mpl * rl * vl + mmr * rr * vr) + p12 * ysn;
    f[3] = c12 * (mpl * rl * wl + mmr * rr * wr) + p12 * zsn;
    f[4] = c12 * (mpl * rl * hl + mmr * rr * hr);
}

/* Ausmpw_Scheme, Flux_Inviscid.cpp:13463-13626: AUSMPW.  It differs from
 * AUSMPW+ above in its sound speeds (gamma p (1 / (rho + SMALL)), mean
 * 1 / (0.5 (a_L + a_R) + SMALL)), in a pressure weight without limiter, and in
 * the pressure corrections, taken for |M| < 1 with no test of p12.  Its split
 * polynomials FMSplit4 / FPSplit5 (:14109-14125) with beta = alpha = 0 are
 * FMmpn / FMppn exactly. */
static void ausmpw_flux(const double *ql, const double *qr, double gl, double gr, double xsn, double ysn,
                        double zsn, double *f)
{
    double rl = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
    double rr = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
    double v2l = ul * ul + vl * vl + wl * wl;
    double v2r = ur * ur + vr * vr + wr * wr;
    double hl = (gl / (gl - 1.0)) * (pl / rl) + 0.5 * v2l;
    double hr = (gr / (gr - 1.0)) * (pr / rr) + 0.5 * v2r;
    double vnl = xsn * ul + ysn * vl + zsn * wl;
    double vnr = xsn * ur + ysn * vr + zsn * wr;
    double orl = 1.0 / (rl + OX_SMALL), orr = 1.0 / (rr + OX_SMALL);
    double cl = sqrt(gl * pl * orl), cr = sqrt(gr * pr * orr);
    double cm = 0.5 * (cl + cr);
    double ocm = 1.0 / (cm + OX_SMALL);
    double ml = vnl * ocm, mr = vnr * ocm;
    double fm4l = fm_mpn(ml, 1.0), fm4r = fm_mpn(mr, -1.0);
    double fp5l = fm_ppn(ml, 1.0), fp5r = fm_ppn(mr, -1.0);
    double m12 = fm4l + fm4r;
    double p12 = fp5l * pl + fp5r * pr;
    double minplr = omin(pl / (pr + OX_SMALL), pr / (pl + OX_SMALL));
    double fw = 1.0 - minplr * minplr * minplr;
    double op12 = 1.0 / (p12 + OX_SMALL);
    double fl = 0.0, fr = 0.0;
    if (fabs(ml) < 1.0) fl = pl * op12 - 1.0;
    if (fabs(mr) < 1.0) fr = pr * op12 - 1.0;
    double mpl, mmr;
    if (m12 >= 0.0) {
        double o = 1.0 + fr;
        mpl = fm4l + fm4r * ((1.0 - fw) * o - fl);
        mmr = fm4r * fw * o;
    } else {
        double o = 1.0 + fl;
        mpl = fm4l * fw * o;
        mmr = fm4r + fm4l * ((1.0 - fw) * o - fr);
    }
    f[0] = cm * (mpl * rl + mmr * rr);
    f[1] = cm * (mpl * rl * ul + mmr * rr * ur) + p12 * xsn;
    f[2] = cm * (mpl * rl * vl + mmr * rr * vr) + p12 * ysn;
    f[3] = cm * (mpl * rl * wl + mmr * rr * wr) + p12 * zsn;
    f[4] = cm * (mpl * rl * hl + mmr * rr * hr);
}

/* PositiveCheckForDensityAndPressure: rho > 0 and p > 0. */
static inline int positive(const double *q) { return q[0] > 0.0 && q[4] > 0.0; }

/* NSSolverUnstruct::InviscidFlux (NSSolverUnstruct.cpp:6912-6973): per face
 * GetQlQr / GetGamaLR (5507-5571), ReConstructFaceValue (13991-14193),
 * BoundaryQlQrFix (13725-13951), the scheme times the face area
 * (InviscidFluxWrap, 14466-14488), LoadFlux (6435-6495).  res is
 * accumulated (callers zero it first, as Controller::LoadResiduals does). */
void ox_inviscid_flux(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                      const double *gama, const double *dqdx, const double *dqdy, const double *dqdz,
                      const double *limit, double *res)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double ql[5], qr[5], tr[5];
        for (int k = 0; k < 5; ++k) { ql[k] = q[k * nt + le]; qr[k] = q[k * nt + re]; }
        if (!p->first_order) {   /* ReConstructFaceValue returns at once in first order (:14014-14021) */
            double lim_l = limit[le], lim_r = limit[re];
            if (p->recon_method == 1) lim_l = lim_r = omin(limit[le], limit[re]);
            double dx = m->xfc[f] - m->xcc[le], dy = m->yfc[f] - m->ycc[le], dz = m->zfc[f] - m->zcc[le];
            for (int k = 0; k < 5; ++k)
                tr[k] = ql[k] + lim_l * (dqdx[k * nt + le] * dx + dqdy[k * nt + le] * dy + dqdz[k * nt + le] * dz);
            if (positive(tr)) for (int k = 0; k < 5; ++k) ql[k] = tr[k];
            dx = m->xfc[f] - m->xcc[re]; dy = m->yfc[f] - m->ycc[re]; dz = m->zfc[f] - m->zcc[re];
            for (int k = 0; k < 5; ++k)
                tr[k] = qr[k] + lim_r * (dqdx[k * nt + re] * dx + dqdy[k * nt + re] * dy + dqdz[k * nt + re] * dz);
            if (positive(tr)) for (int k = 0; k < 5; ++k) qr[k] = tr[k];
        }
        double xn = m->xfn[f], yn = m->yfn[f], zn = m->zfn[f];
        if (f < nb) {
            int t = g->region_type[g->bface_region[f]];
            if (t == OX_BC_SOLID_SURFACE || t == OX_BC_SYMMETRY) {
                for (int k = 0; k < 5; ++k) { double a = 0.5 * (q[k * nt + le] + q[k * nt + re]); ql[k] = qr[k] = a; }
                if (t == OX_BC_SYMMETRY) {
                    double vn = 2.0 * (xn * ql[1] + yn * ql[2] + zn * ql[3]);
                    qr[1] = ql[1] - vn * xn; qr[2] = ql[2] - vn * yn; qr[3] = ql[3] - vn * zn;
                } else if (p->viscous) {
                    ql[1] = ql[2] = ql[3] = 0.0;
                    qr[1] = qr[2] = qr[3] = 0.0;
                }
            }
        }
        double fl[5];
        switch (p->scheme) {
        case OX_SCHEME_AUSMPW_PLUS: ausmpwp_flux(ql, qr, gama[le], gama[re], xn, yn, zn, p->ausmpw_limiter, fl); break;
        case OX_SCHEME_STEGER: steger_flux(ql, qr, gama[le], gama[re], xn, yn, zn, fl); break;
        case OX_SCHEME_VANLEER: vanleer_flux(ql, qr, gama[le], gama[re], xn, yn, zn, fl); break;
        case OX_SCHEME_VANLEER_ROTATE: vanleer_rotate_flux(ql, qr, gama[le], gama[re], xn, yn, zn, fl); break;
        case OX_SCHEME_HLLE: hlle_flux(ql, qr, gama[le], gama[re], xn, yn, zn, fl); break;
        case OX_SCHEME_AUSMDV: ausmdv_flux(ql, qr, gama[le], gama[re], xn, yn, zn, fl); break;
        case OX_SCHEME_AUSMPW: ausmpw_flux(ql, qr, gama[le], gama[re], xn, yn, zn, fl); break;
        default: roe_flux(ql, qr, gama[le], gama[re], xn, yn, zn, p->entropy_acoustic, p->entropy_convective, fl);
        }
        for (int k = 0; k < 5; ++k) {
            double fa = fl[k] * m->area[f];
            res[k * nt + le] -= fa;
            if (f >= nb) res[k * nt + re] += fa;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Viscous terms                                                             */
/* ------------------------------------------------------------------------ */

/* ComputeViscousCoefficientWithoutChemical, NSSolverUnstruct.cpp:6722-6747
 * (Sutherland, every cell and ghost); laminar runs have zero eddy viscosity. */
void ox_viscosity(const ox_grid *g, const ox_params *p, const double *t, double *visl, double *vist)
{
    int nt = ntot(g);
    double s = p->tsuth_nd;
    for (int c = 0; c < nt; ++c) {
        visl[c] = t[c] * sqrt(t[c]) * (1.0 + s) / (t[c] + s);
        if (p->viscous == 1) vist[c] = 0.0;
    }
}

/* NSSolverUnstruct::ViscousFlux (7058-7110) per face, in face order:
 * UnstructGrid::FaceWeight (Geo_UnstructGrid.cpp:2420-2478), GetVisFaceValue
 * (NSSolverUnstruct.cpp:7126-7375; static adiabatic walls), ComputeVisflux
 * (12977-13378; perfect gas, no Reynolds-stress model), LoadFlux.  res is
 * accumulated after the inviscid flux. */
void ox_viscous_flux(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, const double *t,
                     const double *visl, const double *vist, const double *dqdx, const double *dqdy,
                     const double *dqdz, const double *dtdx, const double *dtdy, const double *dtdz, double *res)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    double ore = 1.0 / p->reynolds;
    double oprl = 1.0 / p->prandtl, oprt = 1.0 / p->prandtl_turb;
    double cp = 1.0 / ((p->gama - 1.0) * (p->mach * p->mach));
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        int bt = f < nb ? g->region_type[g->bface_region[f]] : 0;
        int wall = f < nb && is_wall(bt);
        /* FaceWeight */
        double dxl = m->xfc[f] - m->xcc[le], dyl = m->yfc[f] - m->ycc[le], dzl = m->zfc[f] - m->zcc[le];
        double dxr = m->xfc[f] - m->xcc[re], dyr = m->yfc[f] - m->ycc[re], dzr = m->zfc[f] - m->zcc[re];
        double d1 = sqrt(dxl * dxl + dyl * dyl + dzl * dzl), d2 = sqrt(dxr * dxr + dyr * dyr + dzr * dzr);
        double dlt = 1.0 / (d1 + d2 + OX_SMALL);
        double dwl = d2 * dlt, dwr = d1 * dlt;
        if (f < nb && bt != OX_BC_INTERFACE) { dwl = 1.0; dwr = 0.0; }   /* FaceWeight, Geo_UnstructGrid.cpp:2475 */
        /* GetVisFaceValue */
        double mul = 0.5 * (visl[le] + visl[re]);
        double mut = 0.5 * (vist[le] + vist[re]);
        double pf[5];
        for (int k = 0; k < 5; ++k) pf[k] = 0.5 * (q[k * nt + le] + q[k * nt + re]);
        double tmf = 0.5 * (t[le] + t[re]);
        double kcp = (mul * oprl + mut * oprt) * cp;
        if (wall) pf[1] = pf[2] = pf[3] = 0.0;
        /* ComputeVisflux */
        double nxs = m->xfn[f], nys = m->yfn[f], nzs = m->zfn[f];
        double t1x, t1y, t1z;
        if (fabs(nxs) > OX_SMALL) { t1x = nys; t1y = -nxs; t1z = 0.0; }
        else if (fabs(nys) > OX_SMALL) { t1x = -nys; t1y = nxs; t1z = 0.0; }
        else if (fabs(nzs) > OX_SMALL) { t1x = 0.0; t1y = -nzs; t1z = nys; }
        else continue;  /* zero flux */
        double on = 1.0 / sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
        t1x *= on; t1y *= on; t1z *= on;
        double t2x = nys * t1z - nzs * t1y, t2y = nzs * t1x - nxs * t1z, t2z = nxs * t1y - nys * t1x;
        double dxL = m->xcc[le] - m->xfc[f], dyL = m->ycc[le] - m->yfc[f], dzL = m->zcc[le] - m->zfc[f];
        double dxR = m->xcc[re] - m->xfc[f], dyR = m->ycc[re] - m->yfc[f], dzR = m->zcc[re] - m->zfc[f];
        double dL = nxs * dxL + nys * dyL + nzs * dzL;
        double dR = nxs * dxR + nys * dyR + nzs * dzR;
        double tmp = -dL / (sqrt(dxL * dxL + dyL * dyL + dzL * dzL) + OX_SMALL);
        tmp = omin(tmp, 1.0); tmp = omax(tmp, -1.0);
        double a1 = asin(tmp) * 180.0 / OX_PI;
        tmp = dR / (sqrt(dxR * dxR + dyR * dyR + dzR * dzR) + OX_SMALL);
        tmp = omin(tmp, 1.0); tmp = omax(tmp, -1.0);
        double a2 = asin(tmp) * 180.0 / OX_PI;
        double dxnL = nxs * dL - dxL, dynL = nys * dL - dyL, dznL = nzs * dL - dzL;
        double dxnR = nxs * dR - dxR, dynR = nys * dR - dyR, dznR = nzs * dR - dzR;
        double f1[5], f2[5], fm[5];
        for (int k = 0; k < 5; ++k) { f1[k] = q[k * nt + le]; f2[k] = q[k * nt + re]; }
        double tL = t[le], tR = t[re];
        for (int k = 0; k < 5; ++k) fm[k] = 0.5 * (f1[k] + f2[k]);
        double tM = 0.5 * (tL + tR);
        if (wall) {
            tM = tmf;
            fm[0] = fm[4] / (p->coef_state * tM);
        }
        if (a1 > p->skewness_angle && a2 > p->skewness_angle) {
            for (int k = 0; k < 5; ++k) {
                f1[k] += dqdx[k * nt + le] * dxnL + dqdy[k * nt + le] * dynL + dqdz[k * nt + le] * dznL;
                f2[k] += dqdx[k * nt + re] * dxnR + dqdy[k * nt + re] * dynR + dqdz[k * nt + re] * dznR;
            }
            tL += dtdx[le] * dxnL + dtdy[le] * dynL + dtdz[le] * dznL;
            tR += dtdx[re] * dxnR + dtdy[re] * dynR + dtdz[re] * dznR;
            if (tL < OX_SMALL) tL = t[le];
            if (tR < OX_SMALL) tR = t[re];
            for (int k = 0; k < 5; ++k) fm[k] = pf[k];
            tM = tmf;
        }
        double dfdn[5] = {0, 0, 0, 0, 0}, dtdn = 0.0;
        if (a1 > 0.0 && a2 > 0.0 && fabs(dL) > OX_TINY && fabs(dR) > OX_TINY) {
            double dtmp = dL * dL + dR * dR;
            double wL = dL * dL / dtmp;
            double wR = 1.0 - wL;
            if (f < nb && bt != OX_BC_INTERFACE) { wL = 1.0; wR = 0.0; }   /* ComputeVisflux :13261 */
            for (int k = 0; k < 5; ++k) {
                double e1 = (f1[k] - fm[k]) / dL, e2 = (f2[k] - fm[k]) / dR;
                dfdn[k] = wL * e1 + wR * e2;
            }
            double dtd1 = (tL - tM) / dL, dtd2 = (tR - tM) / dR;
            dtdn = dtd1 * wL + dtd2 * wR;
        }
        double gx[5], gy[5], gz[5];
        for (int k = 1; k <= 3; ++k) {
            double fx = dwl * dqdx[k * nt + le] + dwr * dqdx[k * nt + re];
            double fy = dwl * dqdy[k * nt + le] + dwr * dqdy[k * nt + re];
            double fz = dwl * dqdz[k * nt + le] + dwr * dqdz[k * nt + re];
            double dt1 = t1x * fx + t1y * fy + t1z * fz;
            double dt2 = t2x * fx + t2y * fy + t2z * fz;
            gx[k] = nxs * dfdn[k] + t1x * dt1 + t2x * dt2;
            gy[k] = nys * dfdn[k] + t1y * dt1 + t2y * dt2;
            gz[k] = nzs * dfdn[k] + t1z * dt1 + t2z * dt2;
        }
        double dudx = gx[1], dudy = gy[1], dudz = gz[1];
        double dvdx = gx[2], dvdy = gy[2], dvdz = gz[2];
        double dwdx = gx[3], dwdy = gy[3], dwdz = gz[3];
        double qn = 0.0;
        qn += kcp * dtdn;
        double div = (2.0 / 3.0) * (dudx + dvdy + dwdz);
        double vis = mul + mut;
        double txx = vis * (2.0 * dudx - div), tyy = vis * (2.0 * dvdy - div), tzz = vis * (2.0 * dwdz - div);
        double txy = vis * (dudy + dvdx), txz = vis * (dudz + dwdx), tyz = vis * (dvdz + dwdy);
        double fv[5];
        fv[0] = 0.0;
        fv[1] = nxs * txx + nys * txy + nzs * txz;
        fv[2] = nxs * txy + nys * tyy + nzs * tyz;
        fv[3] = nxs * txz + nys * tyz + nzs * tzz;
        fv[4] = fm[1] * fv[1] + fm[2] * fv[2] + fm[3] * fv[3] + qn;
        for (int k = 0; k < 5; ++k) {
            double fl = -ore * m->area[f] * fv[k];
            res[k * nt + le] -= fl;
            if (f >= nb) res[k * nt + re] += fl;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Spectral radius and time step                                             */
/* ------------------------------------------------------------------------ */

/* SpectrumRadiusInviscid, NSSolverUnstruct.cpp:5749-5850; the viscous part
 * (SpectrumRadiusViscous, 5852-5940) is added for viscous runs. */
void ox_spectrum(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                 const double *gama, const double *visl, const double *vist, double *inv_spec, double *vis_spec)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    for (int c = 0; c < nc; ++c) { inv_spec[c] = 0.0; if (vis_spec) vis_spec[c] = 0.0; }
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double xn = m->xfn[f], yn = m->yfn[f], zn = m->zfn[f];
        double vnl = xn * q[nt + le] + yn * q[2 * nt + le] + zn * q[3 * nt + le];
        double vnr = xn * q[nt + re] + yn * q[2 * nt + re] + zn * q[3 * nt + re];
        double gm = 0.5 * (gama[le] + gama[re]);
        double pm = 0.5 * (q[4 * nt + le] + q[4 * nt + re]);
        double rm = 0.5 * (q[le] + q[re]);
        double vn = 0.5 * (vnl + vnr);
        double cm = sqrt(gm * pm / rm);
        double s = 0.5 * m->area[f] * (fabs(vn) + cm);
        inv_spec[le] += s;
        if (re < nc) inv_spec[re] += s;
    }
    if (!p->viscous || !vis_spec) return;
    /* visSpetrumMethod 2 (5930-5960): 2 mu / (rho |n.dr| Re) * A/2 */
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double dx = m->xcc[re] - m->xcc[le], dy = m->ycc[re] - m->ycc[le], dz = m->zcc[re] - m->zcc[le];
        double ds = fabs(m->xfn[f] * dx + m->yfn[f] * dy + m->zfn[f] * dz);
        double mul = 0.5 * (visl[le] + visl[re]);
        double mut = 0.5 * (vist[le] + vist[re]);
        double rho = 0.5 * (q[le] + q[re]);
        double vs = 2.0 * (mul + mut) / (rho * ds * p->reynolds + OX_SMALL);
        vs *= 0.5 * m->area[f];
        vis_spec[le] += vs;
        if (re < nc) vis_spec[re] += vs;
    }
}

/* NSSolver::ComputeCFL, CFD/NSSolver/src/NSSolver.cpp:595-668 (cflMethod 0,
 * single grid level: the outer step drives the ramp). */
double ox_cfl(const ox_params *p, int step)
{
    if (step >= p->cfl_vary_step) return p->cfl_end;
    return p->cfl_start + (p->cfl_end - p->cfl_start) * step / p->cfl_vary_step;
}

/* LocalTimeStep + LimitCFL (NSSolverUnstruct.cpp:5999-6118),
 * Controller::ComputeMinTimeStep / ReduceMaxTimeStep (Controller.cpp:706-788,
 * NSSolverUnstruct.cpp:5696-5745): dt = CFL_cell vol / spec, clamped to
 * ktmax * min(dt), divided by vol; ghosts copy the owner. */
double ox_timestep_raw(const ox_grid *g, const ox_metrics *m, const ox_params *p, int step, const double *q,
                       const double *inv_spec, const double *vis_spec, double *dt)
{
    int nt = ntot(g), nc = g->n_cell;
    double cfl = ox_cfl(p, step);
    double plo = 0.001 * p->p_total, phi = 0.02 * p->p_total;
    double mindt = OX_LARGE;
    for (int c = 0; c < nc; ++c) {
        double cc = cfl;
        double pc = q[4 * nt + c];
        if (pc < plo) cc = p->cfl_start;
        else if (pc < phi) cc = (pc - phi) * (cfl - p->cfl_start) / (phi - plo) + cfl;
        if (m->skew[c] < 0.1) cc *= 0.1;
        else if (m->skew[c] < 10.0) cc *= (1.0 - exp(0.0 - m->skew[c]));
        double spec = inv_spec[c];
        if (p->viscous) spec += vis_spec[c];
        dt[c] = cc * m->vol[c] / spec;
        mindt = omin(mindt, dt[c]);
    }
    return mindt;
}

void ox_timestep_clamp(const ox_grid *g, const ox_metrics *m, const ox_params *p, double mindt, double *dt)
{
    int nc = g->n_cell;
    for (int c = 0; c < nc; ++c) {
        if (p->ktmax > 0) dt[c] = omin(dt[c], p->ktmax * mindt);
        dt[c] /= m->vol[c];
    }
    for (int f = 0; f < g->n_bface; ++f) dt[nc + f] = dt[g->left[f]];
}

void ox_timestep(const ox_grid *g, const ox_metrics *m, const ox_params *p, int step, const double *q,
                 const double *inv_spec, const double *vis_spec, double *dt)
{
    ox_timestep_clamp(g, m, p, ox_timestep_raw(g, m, p, step, q, inv_spec, vis_spec, dt), dt);
}

/* ------------------------------------------------------------------------ */
/* LU-SGS                                                                    */
/* ------------------------------------------------------------------------ */

/* RoeAveragedVariables, API/Physics/src/Flux_Inviscid.cpp:15440-15465. */
static void roe_average(const double *a, double ga, const double *b, double gb, double *o)
{
    double hL = ga / (ga - 1.0) * a[4] / a[0] + 0.5 * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
    double hR = gb / (gb - 1.0) * b[4] / b[0] + 0.5 * (b[1] * b[1] + b[2] * b[2] + b[3] * b[3]);
    double t0 = sqrt(b[0] / a[0]);
    double t1 = 1.0 / (1.0 + t0);
    o[0] = sqrt(b[0] * a[0]);
    o[1] = (a[1] + b[1] * t0) * t1;
    o[2] = (a[2] + b[2] * t0) * t1;
    o[3] = (a[3] + b[3] * t0) * t1;
    double hm = (hL + hR * t0) * t1;
    o[4] = o[0] * (hm - 0.5 * (o[1] * o[1] + o[2] * o[2] + o[3] * o[3])) * (ga - 1.0) / ga;
}

/* MXDQ_STD, API/Physics/src/Jacobian.cpp:13-86 (static grid, ipn = -1) with
 * PerfectGas::ComputeTotalEnthalpyAndDH (PerfectGas.cpp:368-395). */
static void mxdq(const double *prim, double nx, double ny, double nz, double area, double gama,
                 const double *dq, double *f, double radius)
{
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double c2 = fabs(gama * pm / rm);
    double cm = sqrt(c2);
    double cits = nx * um + ny * vm + nz * wm;
    double ipnrad = -radius / omax(OX_SMALL, area);
    double l1 = 0.5 * (cits + ipnrad);
    double l2 = 0.5 * (cits + cm + ipnrad);
    double l3 = 0.5 * (cits - cm + ipnrad);
    double x1 = (l1 + l1 - l2 - l3) / (c2 + c2);
    double x2 = (l2 - l3) / (cm + cm);
    double dc = cits * dq[0] - nx * dq[1] - ny * dq[2] - nz * dq[3];
    double c2dc = c2 * dc;
    double v2 = um * um + vm * vm + wm * wm;
    double g1 = gama - 1.0;
    double dh = -g1 * (um * dq[1] + vm * dq[2] + wm * dq[3] - dq[4]);
    dh += 0.5 * g1 * v2 * dq[0];
    double hm = (gama / g1) * (pm / rm) + 0.5 * v2;
    double a = dh * x1 + dc * x2;
    double b = c2dc * x1 + dh * x2;
    f[0] = (l1 * dq[0] - a) * area;
    f[1] = (l1 * dq[1] - um * a + nx * b) * area;
    f[2] = (l1 * dq[2] - vm * a + ny * b) * area;
    f[3] = (l1 * dq[3] - wm * a + nz * b) * area;
    f[4] = (l1 * dq[4] - hm * a + cits * b) * area;
}

/* Contribution of the neighbour across face f to the sweep of cell c
 * (SolveLUSGSForward body, NSSolverUnstruct.cpp:15251-15370). */
static void lusgs_face(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                       const double *gama, const double *visl, const double *vist, const double *dq, int c, int f,
                       double *df)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    int le = g->left[f], re = f < nb ? nc + f : g->right[f];
    double nx = m->xfn[f], ny = m->yfn[f], nz = m->zfn[f];
    if (re == c) { int s = le; le = re; re = s; nx = -nx; ny = -ny; nz = -nz; }
    double ql[5], qn[5], dqn[5], fp[5];
    for (int k = 0; k < 5; ++k) { ql[k] = q[k * nt + le]; qn[k] = q[k * nt + re]; dqn[k] = dq[k * nt + re]; }
    roe_average(ql, gama[le], qn, gama[re], fp);
    double gm = gama[re];
    double vn = nx * fp[1] + ny * fp[2] + nz * fp[3];
    double rad = (fabs(vn) + sqrt(gm * fp[4] / fp[0])) * m->area[f];
    mxdq(qn, nx, ny, nz, m->area[f], gm, dqn, df, rad);
    if (p->viscous) {
        double dist = fabs(m->xfn[f] * (m->xcc[re] - m->xcc[le]) + m->yfn[f] * (m->ycc[re] - m->ycc[le]) +
                           m->zfn[f] * (m->zcc[re] - m->zcc[le]));
        double mul = 0.5 * (visl[le] + visl[re]);
        double mut = 0.5 * (vist[le] + vist[re]);
        double rho = 0.5 * (q[le] + q[re]);
        double vs = 2.0 * (mul + mut) / (rho * dist * p->reynolds + OX_SMALL);
        vs *= 0.5 * m->area[f];
        for (int k = 0; k < 5; ++k) df[k] -= vs * dqn[k];
    }
}

/* SetGhostDQLUSGS (NSSolverUnstruct.cpp:14767-14810) with
 * SetSymmBCGhostDQLUSGS (14812-14915) and SetWallBCGhostDQLUSGS (14917-15006);
 * far field: zero. */
static void ghost_dq(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                     const double *gama, double *dq)
{
    int nt = ntot(g), nc = g->n_cell;
    for (int f = 0; f < g->n_bface; ++f) {
        int t = g->region_type[g->bface_region[f]];
        int le = g->left[f], re = nc + f;
        if (t == OX_BC_SYMMETRY || (is_wall(t) && !p->viscous)) {
            double r = q[le], u = q[nt + le], v = q[2 * nt + le], w = q[3 * nt + le], pp = q[4 * nt + le];
            double em = (pp / r) / (gama[le] - 1.0) + 0.5 * (u * u + v * v + w * w);
            double Q[5] = {r, r * u, r * v, r * w, r * em};
            for (int k = 0; k < 5; ++k) Q[k] += dq[k * nt + le];
            double rm = q[re], um = q[nt + re], vm = q[2 * nt + re], wm = q[3 * nt + re], pm = q[4 * nt + re];
            double xn = m->xfn[f], yn = m->yfn[f], zn = m->zfn[f];
            dq[re] = dq[le];
            double rvn = 2.0 * (xn * dq[nt + le] + yn * dq[2 * nt + le] + zn * dq[3 * nt + le]);
            dq[nt + re] = dq[nt + le] - xn * rvn;
            dq[2 * nt + re] = dq[2 * nt + le] - yn * rvn;
            dq[3 * nt + re] = dq[3 * nt + le] - zn * rvn;
            rvn = 2.0 * (xn * Q[1] + yn * Q[2] + zn * Q[3]);
            double ru = Q[1] - xn * rvn, rv = Q[2] - yn * rvn, rw = Q[3] - zn * rvn;
            double pnew = Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / Q[0];
            double g1 = gama[le] - 1.0;
            dq[4 * nt + re] = pnew - pm / g1 + 0.5 * ((ru * ru + rv * rv + rw * rw) / Q[0] - rm * (um * um + vm * vm + wm * wm));
        } else if (is_wall(t)) {
            dq[re] = dq[le];
            dq[nt + re] = -dq[nt + le];
            dq[2 * nt + re] = -dq[2 * nt + le];
            dq[3 * nt + re] = -dq[3 * nt + le];
            dq[4 * nt + re] = dq[4 * nt + le];
        } else {
            for (int k = 0; k < 5; ++k) dq[k * nt + re] = 0.0;
        }
    }
}

static double *lusgs_diag(const ox_grid *g, const ox_params *p, const double *dt, const double *inv_spec,
                          const double *vis_spec)
{
    double *diag = malloc(sizeof(double) * g->n_cell);
    for (int c = 0; c < g->n_cell; ++c) {
        diag[c] = 1.0 / dt[c] + inv_spec[c];
        if (p->viscous) diag[c] += vis_spec[c];
    }
    return diag;
}

/* SolveLUSGSForward (NSSolverUnstruct.cpp:15118-15444): lower neighbours
 * j < i over interior faces; then SetGhostDQLUSGS (:15428). */
static double sweep_forward(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                            const double *gama, const double *visl, const double *vist, const double *res,
                            const double *diag, double *dq, double *dflux)
{
    int nt = ntot(g), nc = g->n_cell;
    double norm = 0.0;
    for (int c = 0; c < nc; ++c) {
        double rhs0[5] = {0, 0, 0, 0, 0}, ux[5], old[5];
        for (int k = 0; k < 5; ++k) {
            old[k] = dq[k * nt + c];
            dq[k * nt + c] = res[k * nt + c];
            ux[k] = dflux[k * nt + c];
            dflux[k * nt + c] = 0.0;
        }
        for (int j = m->c2f_off[c]; j < m->c2f_off[c + 1]; ++j) {
            int f = m->c2f[j];
            if (f < g->n_bface) continue;
            int le = g->left[f], re = g->right[f];
            if (le > c || re > c) continue;
            double df[5];
            lusgs_face(g, m, p, q, gama, visl, vist, dq, c, f, df);
            for (int k = 0; k < 5; ++k) rhs0[k] += df[k];
        }
        for (int k = 0; k < 5; ++k) {
            double v = (dq[k * nt + c] - ux[k] - rhs0[k]) / diag[c];
            dflux[k * nt + c] += rhs0[k];
            dq[k * nt + c] = v;
            norm += (v - old[k]) * (v - old[k]);
        }
    }
    ghost_dq(g, m, p, q, gama, dq);
    return norm;
}

/* SolveLUSGSBackward (NSSolverUnstruct.cpp:15446-15690): upper neighbours
 * j > i, boundary ghosts included. */
static double sweep_backward(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                             const double *gama, const double *visl, const double *vist, const double *res,
                             const double *diag, double *dq, double *dflux)
{
    int nt = ntot(g), nc = g->n_cell;
    double norm = 0.0;
    for (int c = nc - 1; c >= 0; --c) {
        double rhs0[5] = {0, 0, 0, 0, 0}, lx[5], old[5];
        for (int k = 0; k < 5; ++k) {
            old[k] = dq[k * nt + c];
            dq[k * nt + c] = res[k * nt + c];
            lx[k] = dflux[k * nt + c];
            dflux[k * nt + c] = 0.0;
        }
        for (int j = m->c2f_off[c]; j < m->c2f_off[c + 1]; ++j) {
            int f = m->c2f[j];
            int le = g->left[f], re = f < g->n_bface ? nc + f : g->right[f];
            if (le < c || re < c) continue;
            double df[5];
            lusgs_face(g, m, p, q, gama, visl, vist, dq, c, f, df);
            for (int k = 0; k < 5; ++k) rhs0[k] += df[k];
        }
        for (int k = 0; k < 5; ++k) {
            double v = (dq[k * nt + c] - lx[k] - rhs0[k]) / diag[c];
            dflux[k * nt + c] += rhs0[k];
            dq[k * nt + c] = v;
            norm += (v - old[k]) * (v - old[k]);
        }
    }
    return norm;
}

/* Controller::LUSGS (Controller.cpp:1878-1955), one or more symmetric sweeps:
 * Diagonal (NSSolverUnstruct.cpp:15867-15935), the forward sweep with
 * SetGhostDQLUSGS, the backward sweep.  dq [5][nTotal] is the output. */
void ox_lusgs(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, const double *gama,
              const double *t, const double *visl, const double *vist, const double *res, const double *dt,
              const double *inv_spec, const double *vis_spec, double *dq)
{
    (void)t;
    int nt = ntot(g);
    double *diag = lusgs_diag(g, p, dt, inv_spec, vis_spec);
    double *dflux = calloc((size_t)5 * nt, sizeof(double));
    /* LUSGSInitialization (Controller.cpp:1732-1785): dq = res for a single
     * sweep (ghost residuals are zero), zero otherwise. */
    for (int i = 0; i < 5 * nt; ++i) dq[i] = p->n_sweeps == 1 ? res[i] : 0.0;
    double norm0 = 0.0;
    for (int sweep = 0; sweep < p->n_sweeps; ++sweep) {
        double norm = sweep_forward(g, m, p, q, gama, visl, vist, res, diag, dq, dflux);
        norm += sweep_backward(g, m, p, q, gama, visl, vist, res, diag, dq, dflux);
        if (sweep == 0) norm0 = norm;
        else if (norm / norm0 < p->lusgs_tol) break;
    }
    free(diag); free(dflux);
}

void ox_lusgs_forward(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                      const double *gama, const double *visl, const double *vist, const double *res,
                      const double *dt, const double *inv_spec, const double *vis_spec, double *dq, double *dflux)
{
    int nt = ntot(g);
    double *diag = lusgs_diag(g, p, dt, inv_spec, vis_spec);
    for (int i = 0; i < 5 * nt; ++i) { dq[i] = res[i]; dflux[i] = 0.0; }
    sweep_forward(g, m, p, q, gama, visl, vist, res, diag, dq, dflux);
    free(diag);
}

void ox_lusgs_backward(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q,
                       const double *gama, const double *visl, const double *vist, const double *res,
                       const double *dt, const double *inv_spec, const double *vis_spec, double *dq, double *dflux)
{
    double *diag = lusgs_diag(g, p, dt, inv_spec, vis_spec);
    sweep_backward(g, m, p, q, gama, visl, vist, res, diag, dq, dflux);
    free(diag);
}

/* ------------------------------------------------------------------------ */
/* Update                                                                    */
/* ------------------------------------------------------------------------ */

/* NSSolverUnstruct::UpdateFlowField (NSSolverUnstruct.cpp:14587-14765) with
 * SolutionFix (14509-14585): in place, cells in ascending order, so a repair
 * sees already-updated lower neighbours.  Returns the repaired-cell count. */
int ox_update(const ox_grid *g, const ox_metrics *m, const ox_params *p, double *q, const double *gama,
              const double *dq)
{
    int nt = ntot(g), nc = g->n_cell, nneg = 0;
    double rlim = 1.0e-6 * p->prim_inf[0], plim = 1.0e-6 * p->prim_inf[4];
    for (int c = 0; c < nc; ++c) {
        double r = q[c], u = q[nt + c], v = q[2 * nt + c], w = q[3 * nt + c], pp = q[4 * nt + c];
        double gm = gama[c];
        double em = (pp / r) / (gm - 1.0) + 0.5 * (u * u + v * v + w * w);
        double Q[5] = {r, r * u, r * v, r * w, r * em};
        for (int k = 0; k < 5; ++k) Q[k] += dq[k * nt + c];
        double prim[5];
        if (Q[0] <= 0.0) {
            prim[0] = Q[0];
            for (int k = 1; k < 5; ++k) prim[k] = q[k * nt + c];
        } else {
            double od = 1.0 / Q[0];
            double um = Q[1] * od, vm = Q[2] * od, wm = Q[3] * od;
            double ie = Q[4] - 0.5 * Q[0] * (um * um + vm * vm + wm * wm);
            prim[0] = Q[0]; prim[1] = um; prim[2] = vm; prim[3] = wm; prim[4] = (gm - 1.0) * ie;
        }
        if (prim[0] < rlim || prim[4] < plim) {
            ++nneg;
            double acc[5] = {0, 0, 0, 0, 0}, wsum = 0.0;
            for (int j = m->c2f_off[c]; j < m->c2f_off[c + 1]; ++j) {
                int f = m->c2f[j];
                int le = g->left[f], re = f < g->n_bface ? nc + f : g->right[f];
                int nbr = (c == le) ? re : le;
                if (q[nbr] < rlim || q[4 * nt + nbr] < plim) continue;
                wsum += 1.0;
                for (int k = 0; k < 5; ++k) {
                    double fv = q[k * nt + nbr];
                    if (k == 0 || k == 4) fv = fabs(fv);
                    acc[k] += fv;
                }
            }
            if (wsum > 0.0) { double o = 1.0 / wsum; for (int k = 0; k < 5; ++k) prim[k] = acc[k] * o; }
            else for (int k = 0; k < 5; ++k) prim[k] = p->prim_inf[k];
        }
        for (int k = 0; k < 5; ++k) q[k * nt + c] = prim[k];
    }
    return nneg;
}

/* Residual monitor, API/Physics/src/Residual.cpp:534-600 and 184-224 (unit
 * grid scale): sqrt(sum res_rho^2 / nCell). */
/* Node values of nv cell fields f [nv][nTotal] and the temperature t
 * (NSSolverUnstruct::ComputeNodeValue, NSSolverUnstruct.cpp:4734-5080, then
 * ModifyNodeValue, :5083-5116): node boundary types by priority (solid wall,
 * then far field, then other non-symmetry boundaries); boundary nodes take
 * 1/distance-weighted face values 0.5 (f_L + f_ghost) of their boundary faces
 * (solid wall faces, then far-field, then other non-symmetry faces, each
 * skipping nodes of a higher-priority type); the other nodes, symmetry nodes
 * included, take 1/distance-weighted values of the cells around them; then
 * each node value is divided by its weight sum (0 where the sum is not
 * above SMALL).  fn is [nv][n_node], tn [n_node]. */
enum { OX_NODE_NO_BC = -1 };
void ox_node_values(const ox_grid *g, const ox_metrics *m, const double *f, int nv, const double *t, double *fn,
                    double *tn)
{
    int nn = g->n_node, nb = g->n_bface, nc = g->n_cell, nt = ntot(g);
    int *nbc = malloc(sizeof(int) * nn);
    double *w = calloc((size_t)nn, sizeof(double));
    for (int i = 0; i < nn; ++i) nbc[i] = OX_NODE_NO_BC;
    for (int k = 0; k < nv; ++k) memset(fn + (size_t)k * nn, 0, sizeof(double) * nn);
    memset(tn, 0, sizeof(double) * nn);
    /* node boundary types */
    for (int r = 0; r < g->n_region; ++r) {
        if (g->region_type[r] != OX_BC_SOLID_SURFACE) continue;
        for (int fc = 0; fc < nb; ++fc) {
            if (g->bface_region[fc] != r) continue;
            for (int j = g->face_off[fc]; j < g->face_off[fc + 1]; ++j) nbc[g->face2node[j]] = OX_BC_SOLID_SURFACE;
        }
    }
    for (int r = 0; r < g->n_region; ++r) {
        if (g->region_type[r] != OX_BC_FARFIELD) continue;
        for (int fc = 0; fc < nb; ++fc) {
            if (g->bface_region[fc] != r) continue;
            for (int j = g->face_off[fc]; j < g->face_off[fc + 1]; ++j) {
                int pt = g->face2node[j];
                if (nbc[pt] == OX_BC_SOLID_SURFACE) continue;
                nbc[pt] = OX_BC_FARFIELD;
            }
        }
    }
    for (int r = 0; r < g->n_region; ++r) {
        int bt = g->region_type[r];
        for (int fc = 0; fc < nb; ++fc) {
            if (g->bface_region[fc] != r) continue;
            if (bt == OX_BC_SOLID_SURFACE || bt == OX_BC_FARFIELD || bt == OX_BC_SYMMETRY) continue;
            for (int j = g->face_off[fc]; j < g->face_off[fc + 1]; ++j) {
                int pt = g->face2node[j];
                if (nbc[pt] == OX_BC_SOLID_SURFACE || nbc[pt] == OX_BC_FARFIELD) continue;
                nbc[pt] = bt;
            }
        }
    }
    /* boundary nodes: steps 1 (solid wall), 2 (far field), 3 (others but symmetry) */
    for (int step = 1; step <= 3; ++step) {
        for (int r = 0; r < g->n_region; ++r) {
            int bt = g->region_type[r];
            int take = step == 1 ? bt == OX_BC_SOLID_SURFACE
                     : step == 2 ? bt == OX_BC_FARFIELD
                     : (bt != OX_BC_SOLID_SURFACE && bt != OX_BC_FARFIELD && bt != OX_BC_SYMMETRY);
            if (!take) continue;
            for (int fc = 0; fc < nb; ++fc) {
                if (g->bface_region[fc] != r) continue;
                int le = g->left[fc], re = nc + fc;
                for (int j = g->face_off[fc]; j < g->face_off[fc + 1]; ++j) {
                    int pt = g->face2node[j];
                    if (step == 2 && nbc[pt] == OX_BC_SOLID_SURFACE) continue;
                    if (step == 3 && (nbc[pt] == OX_BC_SOLID_SURFACE || nbc[pt] == OX_BC_FARFIELD)) continue;
                    double dx = g->x[pt] - m->xfc[fc], dy = g->y[pt] - m->yfc[fc], dz = g->z[pt] - m->zfc[fc];
                    double wt = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
                    for (int k = 0; k < nv; ++k) {
                        const double *fk = f + (size_t)k * nt;
                        double qf = 0.5 * (fk[le] + fk[re]);
                        fn[(size_t)k * nn + pt] += qf * wt;
                    }
                    tn[pt] += 0.5 * (t[le] + t[re]) * wt;
                    w[pt] += wt;
                }
            }
        }
    }
    /* step 4: the other nodes from the cells around them */
    for (int c = 0; c < nc; ++c) {
        for (int j = g->cell_off[c]; j < g->cell_off[c + 1]; ++j) {
            int pt = g->cell2node[j];
            if (nbc[pt] != OX_NODE_NO_BC) continue;
            double dx = g->x[pt] - m->xcc[c], dy = g->y[pt] - m->ycc[c], dz = g->z[pt] - m->zcc[c];
            double wt = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
            for (int k = 0; k < nv; ++k) fn[(size_t)k * nn + pt] += f[(size_t)k * nt + c] * wt;
            tn[pt] += t[c] * wt;
            w[pt] += wt;
        }
    }
    for (int i = 0; i < nn; ++i) {
        if (w[i] > OX_SMALL) {
            for (int k = 0; k < nv; ++k) fn[(size_t)k * nn + i] /= w[i];
            tn[i] /= w[i];
        } else {
            for (int k = 0; k < nv; ++k) fn[(size_t)k * nn + i] = 0.0;
            tn[i] = 0.0;
        }
    }
    free(nbc);
    free(w);
}

/* UnstructGrid::CompGradientGGNode_NEW, Geo_UnstructGrid.cpp:4202-4309: face
 * values are the averages of the face's node values, except on boundary faces
 * other than symmetry, which take 0.5 (f_L + f_ghost); divided by the volume;
 * ghost gradients copy the owner's. */
void ox_gradient_ggnode(const ox_grid *g, const ox_metrics *m, const double *q, const double *qn, double *dx,
                        double *dy, double *dz)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    for (int c = 0; c < nt; ++c) dx[c] = dy[c] = dz[c] = 0.0;
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double qf;
        if (f >= nb || g->region_type[g->bface_region[f]] == OX_BC_SYMMETRY) {
            qf = 0.0;
            for (int j = g->face_off[f]; j < g->face_off[f + 1]; ++j) qf += qn[g->face2node[j]];
            qf /= (g->face_off[f + 1] - g->face_off[f]);
        } else {
            qf = 0.5 * (q[le] + q[re]);
        }
        double nx = m->xfn[f] * m->area[f], ny = m->yfn[f] * m->area[f], nz = m->zfn[f] * m->area[f];
        dx[le] += qf * nx; dy[le] += qf * ny; dz[le] += qf * nz;
        if (f >= nb) { dx[re] -= qf * nx; dy[re] -= qf * ny; dz[re] -= qf * nz; }
    }
    for (int c = 0; c < nc; ++c) {
        dx[c] /= m->vol[c]; dy[c] /= m->vol[c]; dz[c] /= m->vol[c];
    }
    for (int f = 0; f < nb; ++f) {
        int le = g->left[f], re = nc + f;
        dx[re] = dx[le]; dy[re] = dy[le]; dz[re] = dz[le];
    }
}

double ox_residual_norm(const ox_grid *g, const double *res)
{
    double s = 0.0;
    for (int c = 0; c < g->n_cell; ++c) s += res[c] * res[c];
    return sqrt(s / g->n_cell);
}

/* One outer iteration (Controller::Relaxation, tscheme = LU_SGS):
 * LoadResiduals, UpdateResiduals (boundary, gamma/T, viscosity, gradient,
 * limiter, inviscid and viscous flux), SpectrumRadius, TimeStep, LUSGS,
 * UpdateFlowField. */
void ox_ns_iteration(const ox_grid *g, const ox_metrics *m, const ox_params *p0, int step, double *q, ox_ns_work *w)
{
    int nt = ntot(g);
    /* Flow initialisation (Simulation::PreSolve, Main/src/Simulation.cpp:1190-1237):
     * isInIniting holds for outer steps 1..flowInitStep.  Then the inviscid flux
     * is Van Leer's (NSSolverUnstruct::ComputeInviscidFlux :14229-14235), the face
     * states are the cell values (ReConstructFaceValue :14014-14021) and the
     * limiter is zero (ComputeLimiter :18203-18224). */
    ox_params pinit = *p0;
    const int init = p0->flow_init_step > 0 && step <= p0->flow_init_step;
    /* the "1st" limiter is first order at every step, with the configured scheme */
    pinit.first_order = init || p0->limiter == OX_LIMITER_FIRST;
    if (init) pinit.scheme = OX_SCHEME_VANLEER;
    const ox_params *p = &pinit;
    ox_gamma_temperature(g, p, q, w->gama, w->t);  /* gama of the ghosts is needed by the far field */
    ox_ns_boundary(g, m, p, q, w->gama);
    ox_gamma_temperature(g, p, q, w->gama, w->t);
    if (p->viscous) ox_viscosity(g, p, w->t, w->visl, w->vist);
    if (p->gradient == 2) {
        /* GG-node.  The reference forms node values in PostSolve, after the
         * update and the boundary (Controller::PostSolve, Controller.cpp:
         * 5063-5205), and SetBoundaryValueOfField (:1467-1491) applies the
         * boundary without recomputing the temperature: the velocity / pressure
         * node values are those of the current state, the temperature node
         * values those of the previous iteration's temperature.  At
         * initialisation (and after a state is loaded) both come from the same
         * state (NSSolver::InitDependentVariables, NSSolver.cpp:757-790). */
        int nn = g->n_node;
        double *qn = malloc(sizeof(double) * 5 * (size_t)nn), *tn = malloc(sizeof(double) * (size_t)nn);
        ox_node_values(g, m, q, 5, w->t, qn, tn);
        const double *tnode = (w->tnode_prev && w->have_tnode_prev) ? w->tnode_prev : tn;
        for (int k = 0; k < 5; ++k)
            ox_gradient_ggnode(g, m, q + (size_t)k * nt, qn + (size_t)k * nn, w->dqdx + (size_t)k * nt,
                               w->dqdy + (size_t)k * nt, w->dqdz + (size_t)k * nt);
        if (p->viscous) ox_gradient_ggnode(g, m, w->t, tnode, w->dtdx, w->dtdy, w->dtdz);
        if (w->qnode) memcpy(w->qnode, qn, sizeof(double) * 5 * (size_t)nn);
        if (w->tnode_prev) {
            memcpy(w->tnode_prev, tn, sizeof(double) * (size_t)nn);
            w->have_tnode_prev = 1;
        }
        free(qn);
        free(tn);
    } else {
        for (int k = 0; k < 5; ++k)
            ox_gradient(g, m, p, q + (size_t)k * nt, w->dqdx + (size_t)k * nt, w->dqdy + (size_t)k * nt,
                        w->dqdz + (size_t)k * nt);
        if (p->viscous) ox_gradient(g, m, p, w->t, w->dtdx, w->dtdy, w->dtdz);
    }
    ox_limiter(g, m, p, q, w->dqdx, w->dqdy, w->dqdz, w->limit);
    memset(w->res, 0, sizeof(double) * 5 * nt);
    ox_inviscid_flux(g, m, p, q, w->gama, w->dqdx, w->dqdy, w->dqdz, w->limit, w->res);
    if (p->viscous)
        ox_viscous_flux(g, m, p, q, w->t, w->visl, w->vist, w->dqdx, w->dqdy, w->dqdz, w->dtdx, w->dtdy, w->dtdz,
                        w->res);
    ox_spectrum(g, m, p, q, w->gama, w->visl, w->vist, w->inv_spec, w->vis_spec);
    ox_timestep(g, m, p, step, q, w->inv_spec, w->vis_spec, w->dt);
    ox_lusgs(g, m, p, q, w->gama, w->t, w->visl, w->vist, w->res, w->dt, w->inv_spec, w->vis_spec, w->dq);
    w->n_negative = ox_update(g, m, p, q, w->gama, w->dq);
    w->res_norm = ox_residual_norm(g, w->res);
    /* Controller::PostSolve (Controller.cpp:5063-5090): ghost states of the
     * updated field, which the turbulence step reads */
    ox_ns_boundary(g, m, p, q, w->gama);
    if (p->viscous == 3) ox_sa_step(g, m, p, q, w);
}

/* ------------------------------------------------------------------------ */
/* Spalart-Allmaras (TurbSolverUnstr, NSMB formation, RANS, no wall function) */
/* ------------------------------------------------------------------------ */

/* PositiveSA, CFD/TurbSolver/include/TurbSolver.h:103-116. */
static double positive_sa(double nue, double visl, double rho)
{
    if (nue < 0.0) {
        double xsi = nue / (visl / rho);
        double xsi3 = xsi * xsi * xsi;
        return nue * (16.0 + xsi3) / (16.0 - xsi3);
    }
    return nue;
}

/* TurbSolverUnstr::Boundary (TurbSolverUnstr.cpp:5919-6019): OutflowBCRegion
 * (copy; symmetry too), WallBCRegion (6116-6160, reflection), FarfieldBCRegion
 * (6546-6640: Riemann-invariant direction picks copy or free stream). */
void ox_sa_boundary(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, const double *gama,
                    double *qt, double *vist)
{
    int nt = ntot(g), nc = g->n_cell;
    const double *pi = p->prim_inf;
    for (int f = 0; f < g->n_bface; ++f) {
        int t = g->region_type[g->bface_region[f]];
        int le = g->left[f], re = nc + f;
        if (t == OX_BC_EXTRAPOLATION || t == OX_BC_SYMMETRY || t == OX_BC_OUTFLOW) {
            vist[re] = vist[le];
            qt[re] = qt[le];
        } else if (is_wall(t)) {
            vist[re] = -vist[le];
            qt[re] = -qt[le];
        } else if (t == OX_BC_FARFIELD) {
            double rin = q[le], uin = q[nt + le], vin = q[2 * nt + le], win = q[3 * nt + le], pin = q[4 * nt + le];
            double vno = m->xfn[f] * pi[1] + m->yfn[f] * pi[2] + m->zfn[f] * pi[3] - 0.0;
            double vni = m->xfn[f] * uin + m->yfn[f] * vin + m->zfn[f] * win - 0.0;
            double vei = sqrt(uin * uin + vin * vin + win * win);
            double ga = gama[le];
            double coo = sqrt(fabs(p->gama * pi[4] / pi[0]));
            double cin = sqrt(fabs(ga * pin / rin));
            int exit_;
            if (vei > cin) {
                exit_ = vni >= 0.0;
            } else {
                double riemp = vni + 2.0 * cin / (ga - 1.0);
                double riemm = vno - 2.0 * coo / (p->gama - 1.0);
                double vnb = 0.5 * (riemp + riemm);
                exit_ = vnb >= 0.0;
            }
            if (exit_) { vist[re] = vist[le]; qt[re] = qt[le]; }
            else { vist[re] = p->vist_inf; qt[re] = p->nut_inf; }
        }
    }
}

/* TurbSolverUnstr::Viscosity, 1eq-sa branch (TurbSolverUnstr.cpp:6910-6960):
 * interior cells only. */
static void sa_viscosity(const ox_grid *g, const double *q, const double *qt, const double *visl, double *vist)
{
    const double cv13 = 7.1 * 7.1 * 7.1;
    for (int c = 0; c < g->n_cell; ++c) {
        double nue = qt[c];
        if (nue > 0.0) {
            double ld = nue * q[c] / (visl[c] + OX_SMALL);
            double ld3 = ld * ld * ld;
            double fv1 = ld3 / (ld3 + cv13);
            vist[c] = q[c] * fv1 * nue;
        } else {
            vist[c] = 0.0;
        }
    }
}

/* SourceFluxOneEquationOriginal (TurbSolverUnstr.cpp:2702-2916), NSMB
 * formation (the cb2 gradient term is carried by the diffusion flux), RANS
 * length scale = wall distance.  Velocity gradients are those of the NS step. */
static void sa_source(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w)
{
    int nt = ntot(g);
    /* (the divergence term cmachfix is computed and zeroed by the reference) */
    const double *dudy = w->dqdy + nt, *dudz = w->dqdz + nt;
    const double *dvdx = w->dqdx + 2 * nt, *dvdz = w->dqdz + 2 * nt;
    const double *dwdx = w->dqdx + 3 * nt, *dwdy = w->dqdy + 3 * nt;
    const double ore = 1.0 / p->reynolds;
    const double karm = 0.41, cb1 = 0.1355, cb2 = 0.622, cv1 = 7.1, cw2 = 0.3, cw3 = 2.0;
    const double sigma = 2.0 / 3.0, sdilim = 1.0e9;
    double kap2 = karm * karm, okap2 = 1.0 / kap2;
    double osigma = 1.0 / sigma;
    double cw1 = cb1 * okap2 + (1.0 + cb2) / sigma;
    double cv13 = cv1 * cv1 * cv1;
    double cw36 = pow(cw3, 6);
    double or6 = 1.0 / 6.0;
    double ct3 = 1.2;
    double saC2 = 0.7, saC3 = 0.9;
    double cb2s = osigma * cb2;
    double cw1kap2 = cw1 * kap2;
    for (int c = 0; c < g->n_cell; ++c) {
        double nue = w->qt[c];
        double omega = sqrt((dwdy[c] - dvdz[c]) * (dwdy[c] - dvdz[c]) + (dudz[c] - dwdx[c]) * (dudz[c] - dwdx[c]) +
                            (dvdx[c] - dudy[c]) * (dvdx[c] - dudy[c]));
        double volume = m->vol[c];
        double olam = q[c] / (w->visl[c] + OX_SMALL);
        double dist2 = m->walldist[c] * m->walldist[c];
        double odist2 = 1.0 / dist2;
        double xsi = nue * olam + OX_SMALL;
        double xsi3 = xsi * xsi * xsi;
        double fv1 = xsi3 / (xsi3 + cv13);
        double fv2 = 1.0 - xsi / (1.0 + xsi * fv1);
        double rs = nue * okap2 * odist2 * ore;
        double nuetrs = nue * rs;
        double sbar = rs * fv2;
        double std_;
        if (sbar >= -saC2 * omega) std_ = omega + sbar;
        else std_ = omega + omega * (saC2 * saC2 * omega + saC3 * sbar) / ((saC3 - 2 * saC2) * omega - sbar);
        double ostd = 1.0 / (std_ + OX_SMALL);
        double r = rs * ostd;
        r = omin(r, 10.0);
        double r5 = pow(r, 5);
        double gg = r + cw2 * (r5 * r - r);
        double g6 = pow(gg, 6);
        double fw = gg * pow((1.0 + cw36) / (g6 + cw36), or6);
        double ft2 = 0.0;
        double grd2 = w->dntx[c] * w->dntx[c] + w->dnty[c] * w->dnty[c] + w->dntz[c] * w->dntz[c];
        double production = cb1 * (1.0 - ft2) * std_ * nue;
        double diffsource = cb2s * grd2 * ore;
        double walldest = (cw1kap2 * fw - cb1 * ft2) * nuetrs;
        double destr_alpha = 50.0;
        if (nue < 0.0) {
            production = cb1 * (1.0 - ct3) * omega * nue;
            walldest = -destr_alpha * cw1kap2 * nuetrs;
        }
        diffsource = omin(sdilim * production, diffsource);
        (void)diffsource;
        double source = production - walldest;
        w->res_t[c] += (source) * volume;
        double dfv2dk = (3.0 * cv13 * pow(fv1 / (xsi + OX_SMALL), 2) - 1.0) / pow(1.0 + xsi * fv1, 2);
        double dsdnu = ore * okap2 * odist2 * (fv2 + xsi * dfv2dk);
        double dfwdg = fw / (gg + OX_SMALL) * (1.0 - g6 / (g6 + cw36));
        double dgdr = 1.0 + cw2 * (6.0 * r5 - 1.0);
        double drdnu = ore * okap2 * odist2 * ostd * (1.0 - nue * ostd * dsdnu);
        double dfwdnu = dfwdg * dgdr * drdnu;
        double prod = cb1 * (1.0 - ft2) * std_;
        double dest = (cw1 * fw - cb1 * ft2 * okap2) * nue * odist2 * ore;
        double prodp = cb1 * ((1.0 - ft2) * dsdnu);
        double destp = (cw1 * (fw + dfwdnu * nue) - cb1 * ft2 * okap2) * odist2 * ore;
        if (nue < 0.0) {
            prod = cb1 * (1.0 - ct3) * omega;
            dest = -destr_alpha * cw1 * nue * odist2 * ore;
            prodp = cb1 * ((1.0 - ct3) * dsdnu);
            destp = -destr_alpha * cw1 * odist2 * ore;
        }
        double prde = prod - dest;
        double prdep = prodp - destp;
        double part1 = -0.5 * (prde - fabs(prde));
        double part2 = -0.5 * (prdep - fabs(prdep)) * nue;
        w->spec_t[c] += (part1 + part2) * volume;
    }
}

/* InviscidFlux: GetQlQrTurbulence / GetQlQrNS (TurbSolverUnstr.cpp:4978-5140,
 * boundary faces averaged; symmetry copies the left nu~) and NNDFlux
 * (5721-5805, first-order upwind, rhoFlag = 0), LoadFlux (2205-2260). */
static void sa_convection(const ox_grid *g, const ox_metrics *m, const double *q, ox_ns_work *w)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double ql = w->qt[le], qr = w->qt[re];
        double pl[4], pr[4];
        for (int k = 0; k < 4; ++k) { pl[k] = q[k * nt + le]; pr[k] = q[k * nt + re]; }
        if (f < nb && g->region_type[g->bface_region[f]] != OX_BC_INTERFACE) {   /* GetQlQr*: :5041, :5125 */
            int t = g->region_type[g->bface_region[f]];
            if (t == OX_BC_SYMMETRY) qr = ql;
            else { double a = 0.5 * (qr + ql); qr = a; ql = a; }
            for (int k = 0; k < 4; ++k) { double a = 0.5 * (pr[k] + pl[k]); pr[k] = a; pl[k] = a; }
        }
        double vnl = m->xfn[f] * pl[1] + m->yfn[f] * pl[2] + m->zfn[f] * pl[3] - 0.0;
        double vnr = m->xfn[f] * pr[1] + m->yfn[f] * pr[2] + m->zfn[f] * pr[3] - 0.0;
        double vnll = 0.5 * (vnl + fabs(vnl));
        double vnrr = 0.5 * (vnr - fabs(vnr));
        double fl = (vnll * ql + vnrr * qr) * m->area[f];
        w->res_t[le] -= fl;
        if (f >= nb) w->res_t[re] += fl;
    }
}

/* ViscousFlux: GetVisFaceValue (TurbSolverUnstr.cpp:3893-3990, mlt of the
 * one-equation branch) and ComputeVisflux, NSMB branch (4438-4674). */
static void sa_diffusion(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w)
{
    int nb = g->n_bface, nc = g->n_cell;
    const double ore = 1.0 / p->reynolds;
    const double cb2 = 0.622, sigma = 2.0 / 3.0, osigma = 1.0 / sigma;
    const double kw_osigma = 1.0 / (2.0 / 3.0);
    const double *qt = w->qt, *visl = w->visl;
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        int t = f < nb ? g->region_type[g->bface_region[f]] : 0;
        /* mlt */
        double nl = qt[le], vl = visl[le], rl = q[le];
        double nr = qt[re], vr = visl[re], rr = q[re];
        if (f < nb) {   /* GetVisFaceValue's mlt loop takes every boundary face alike, interface faces too (:3990-4003) */
            if (nl < 0.0) {
                nl = positive_sa(nl, vl, rl);
                if (is_wall(t)) nr = -nl;
            }
        } else {
            nl = positive_sa(nl, vl, rl);
            nr = positive_sa(nr, vr, rr);
        }
        double mlt = kw_osigma * 0.5 * (vl / rl + vr / rr + nl + nr);
        /* normal derivative */
        double nxs = m->xfn[f], nys = m->yfn[f], nzs = m->zfn[f];
        double dxL = m->xcc[le] - m->xfc[f], dyL = m->ycc[le] - m->yfc[f], dzL = m->zcc[le] - m->zfc[f];
        double dxR = m->xcc[re] - m->xfc[f], dyR = m->ycc[re] - m->yfc[f], dzR = m->zcc[re] - m->zfc[f];
        double dL = nxs * dxL + nys * dyL + nzs * dzL;
        double dR = nxs * dxR + nys * dyR + nzs * dzR;
        double tmp = -dL / (sqrt(dxL * dxL + dyL * dyL + dzL * dzL) + OX_SMALL);
        tmp = omin(tmp, 1.0); tmp = omax(tmp, -1.0);
        double a1 = asin(tmp) * 180.0 / OX_PI;
        tmp = dR / (sqrt(dxR * dxR + dyR * dyR + dzR * dzR) + OX_SMALL);
        tmp = omin(tmp, 1.0); tmp = omax(tmp, -1.0);
        double a2 = asin(tmp) * 180.0 / OX_PI;
        double f1 = qt[le], f2 = qt[re];
        double fm = 0.5 * (f1 + f2);
        double dfdn = 0.0;
        if (a1 > p->turb_skew_angle && a2 > p->turb_skew_angle && fabs(dL) > OX_TINY && fabs(dR) > OX_TINY) {
            double d1 = (f1 - fm) / dL, d2 = (f2 - fm) / dR;
            double dtmp = dL * dL + dR * dR;
            double wl = dL * dL / dtmp;
            double wr = 1.0 - wl;
            dfdn = wl * d1 + wr * d2;
            if (f < nb && t != OX_BC_SYMMETRY && t != OX_BC_INTERFACE) {   /* ComputeVisflux :4569 */
                double nd = (m->xcc[re] - m->xcc[le]) * nxs + (m->ycc[re] - m->ycc[le]) * nys +
                            (m->zcc[re] - m->zcc[le]) * nzs;
                dfdn = (f2 - f1) / nd;
            }
        }
        double flux1 = -ore * (1.0 + cb2) * mlt * dfdn * m->area[f];
        double flux2 = ore * cb2 * osigma * dfdn * m->area[f];
        double nuel = positive_sa(qt[le], visl[le], q[le]);
        double nuer = positive_sa(qt[re], visl[re], q[re]);
        w->res_t[le] -= flux1;
        w->res_t[le] -= flux2 * (visl[le] / q[le] + nuel);
        if (f >= nb) {
            w->res_t[re] += flux1;
            w->res_t[re] += flux2 * (visl[re] / q[re] + nuer);
        }
    }
}

/* SpectrumRadiusOfOneEquation, NSMB branch (TurbSolverUnstr.cpp:4690-4855):
 * upwind convective Jacobians and the diffusion term into spec_turb and the
 * face matrices mat_turbl / mat_turbr (called by Diagonal before the sweeps). */
static void sa_spectrum(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    const double ore = 1.0 / p->reynolds;
    const double sigma = 2.0 / 3.0, osigma = 1.0 / sigma, cb2 = 0.622;
    const double *qt = w->qt, *visl = w->visl;
    double *spec = w->spec_t;
    for (int f = 0; f < g->n_face; ++f) {
        int le = g->left[f], re = f < nb ? nc + f : g->right[f];
        double rl = q[le], ul = q[nt + le], vl = q[2 * nt + le], wl = q[3 * nt + le];
        double vnl = m->xfn[f] * ul + m->yfn[f] * vl + m->zfn[f] * wl - 0.0;
        double ijl = vnl > 0.0 ? rl * vnl * m->area[f] : 0.0;
        double rr = q[re], ur = q[nt + re], vr = q[2 * nt + re], wr = q[3 * nt + re];
        double vnr = m->xfn[f] * ur + m->yfn[f] * vr + m->zfn[f] * wr - 0.0;
        double ijr = vnr < 0.0 ? rr * vnr * m->area[f] : 0.0;
        spec[le] += ijl;
        spec[re] -= ijr;
        w->matr[f] = ijr;
        w->matl[f] = -ijl;
        double orl = 1.0 / (rl + OX_SMALL), orr = 1.0 / (rr + OX_SMALL);
        double nuel = positive_sa(qt[le], visl[le], rl);
        double nuer = positive_sa(qt[re], visl[re], rr);
        if (f < nb && is_wall(g->region_type[g->bface_region[f]])) nuer = -nuel;
        double effl = visl[le] * orl + fabs(nuel);
        double effr = visl[re] * orr + fabs(nuer);
        double eff = 0.5 * (effl + effr);
        double volume = 0.5 * (m->vol[le] + m->vol[re]);
        double ovol = 1.0 / volume;
        double ns2 = m->area[f] * m->area[f];
        spec[le] += ore * ovol * (1.0 + cb2) * (osigma * eff * ns2);
        spec[re] += ore * ovol * (1.0 + cb2) * (osigma * eff * ns2);
        w->matl[f] += -ore * ovol * (1.0 + cb2) * (osigma * eff * ns2);
        w->matr[f] += -ore * ovol * (1.0 + cb2) * (osigma * eff * ns2);
        double cl = cb2 * osigma * effl, cr = cb2 * osigma * effr;
        w->matl[f] += ore * ovol * ns2 * cl;
        w->matr[f] += ore * ovol * ns2 * cr;
    }
}

/* Scalar LU-SGS (SolveLUSGSForward / Backward, TurbSolverUnstr.cpp:1400-1638)
 * with dq initialised by res (Controller::LUSGSInitialization); ghost dq keep
 * the (zero) ghost residual.  Then UpdateFlowField (1180-1230, RANS, no
 * clipping). */
static void sa_sweep_forward(const ox_grid *g, const ox_metrics *m, ox_ns_work *w, double *dfl)
{
    int nt = ntot(g), nb = g->n_bface, nc = g->n_cell;
    double *dq = w->dqt;
    for (int i = 0; i < nt; ++i) { dq[i] = w->res_t[i]; dfl[i] = 0.0; }
    for (int c = 0; c < nc; ++c) {
        double rhs0 = 0.0;
        double ux = dfl[c];
        dfl[c] = 0.0;
        double d = w->res_t[c];
        for (int j = m->c2f_off[c]; j < m->c2f_off[c + 1]; ++j) {
            int f = m->c2f[j];
            int le = g->left[f], re = f < nb ? nc + f : g->right[f];
            if (le > c || re > c) continue;
            double df = (re == c) ? w->matl[f] * dq[le] : w->matr[f] * dq[re];
            rhs0 += df;
        }
        dq[c] = (d - ux - rhs0) / w->spec_t[c];
        dfl[c] += rhs0;
    }
}

static void sa_sweep_backward(const ox_grid *g, const ox_metrics *m, ox_ns_work *w, double *dfl)
{
    int nb = g->n_bface, nc = g->n_cell;
    double *dq = w->dqt;
    for (int c = nc - 1; c >= 0; --c) {
        double rhs0 = 0.0;
        double lx = dfl[c];
        dfl[c] = 0.0;
        double d = w->res_t[c];
        for (int j = m->c2f_off[c]; j < m->c2f_off[c + 1]; ++j) {
            int f = m->c2f[j];
            int le = g->left[f], re = f < nb ? nc + f : g->right[f];
            if (le < c || re < c) continue;
            double df = (re == c) ? w->matl[f] * dq[le] : w->matr[f] * dq[re];
            rhs0 += df;
        }
        dq[c] = (d - lx - rhs0) / w->spec_t[c];
        dfl[c] += rhs0;
    }
    for (int c = 0; c < nc; ++c) w->qt[c] += dq[c];
}

void ox_sa_lusgs_forward(const ox_grid *g, const ox_metrics *m, ox_ns_work *w, double *dfl)
{
    sa_sweep_forward(g, m, w, dfl);
}

void ox_sa_lusgs_backward(const ox_grid *g, const ox_metrics *m, ox_ns_work *w, double *dfl)
{
    sa_sweep_backward(g, m, w, dfl);
}

/* Node values of nu~ (TurbSolverUnstr::ComputeQTurbNodeValue,
 * TurbSolverUnstr.cpp:3480-3814, then ModifyQTurbNodeValue :3816-3845): every
 * face adds its owner's and its other side's value to each of its nodes
 * (boundary faces region by region, reading the face-to-node list at a
 * running position, then the interior faces); the nodes of symmetry, then
 * far-field, then solid-wall faces are reset and take those faces' values
 * only; each node divides by its number of values. */
void ox_qturb_node_values(const ox_grid *g, const double *qt, double *qn)
{
    int nn = g->n_node, nb = g->n_bface, nc = g->n_cell, nf = g->n_face;
    double *acc = calloc((size_t)nn, sizeof(double));
    int *cnt = calloc((size_t)nn, sizeof(int));
    int pos = 0;
    for (int r = 0; r < g->n_region; ++r)
        for (int f = 0; f < nb; ++f) {
            if (g->bface_region[f] != r) continue;
            int le = g->left[f], re = nc + f, n = g->face_off[f + 1] - g->face_off[f];
            for (int j = 0; j < n; ++j) {
                int pt = g->face2node[pos + j];
                acc[pt] += qt[le]; cnt[pt] += 1;
                acc[pt] += qt[re]; cnt[pt] += 1;
            }
            pos += n;
        }
    for (int f = nb; f < nf; ++f) {
        int le = g->left[f], re = g->right[f], n = g->face_off[f + 1] - g->face_off[f];
        for (int j = 0; j < n; ++j) {
            int pt = g->face2node[pos + j];
            acc[pt] += qt[le]; cnt[pt] += 1;
            acc[pt] += qt[re]; cnt[pt] += 1;
        }
        pos += n;
    }
    const int order[3] = {OX_BC_SYMMETRY, OX_BC_FARFIELD, OX_BC_SOLID_SURFACE};
    for (int k = 0; k < 3; ++k) {
        pos = 0;
        for (int r = 0; r < g->n_region; ++r)
            for (int f = 0; f < nb; ++f) {
                if (g->bface_region[f] != r) continue;
                int n = g->face_off[f + 1] - g->face_off[f];
                if (g->region_type[r] == order[k])
                    for (int j = 0; j < n; ++j) { acc[g->face2node[pos + j]] = 0.0; cnt[g->face2node[pos + j]] = 0; }
                pos += n;
            }
        pos = 0;
        for (int r = 0; r < g->n_region; ++r)
            for (int f = 0; f < nb; ++f) {
                if (g->bface_region[f] != r) continue;
                int le = g->left[f], re = nc + f, n = g->face_off[f + 1] - g->face_off[f];
                if (g->region_type[r] == order[k])
                    for (int j = 0; j < n; ++j) {
                        int pt = g->face2node[pos + j];
                        acc[pt] += qt[le]; cnt[pt] += 1;
                        acc[pt] += qt[re]; cnt[pt] += 1;
                    }
                pos += n;
            }
    }
    for (int i = 0; i < nn; ++i) qn[i] = cnt[i] != 0 ? acc[i] / cnt[i] : 0.0;
    free(acc);
    free(cnt);
}

void ox_sa_gradient_phase(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w)
{
    int nt = ntot(g);
    /* LoadResiduals: res = -rhs = -0 */
    for (int i = 0; i < nt; ++i) w->res_t[i] = -0.0;
    /* Controller::UpdateResiduals: SetBoundaryValueOfField, UpdateIndependentField
     * (Viscosity, gradient of nu~) */
    /* GG-node: the nu~ node values are those the previous PostSolve formed
     * after the update and the boundary, or, first, those of the state as
     * initialised or loaded, before any boundary (TurbSolver::
     * InitDependentVariables, TurbSolver.cpp:46-56) */
    if (p->gradient == 2 && w->qtnode && !w->have_qtnode) {
        ox_qturb_node_values(g, w->qt, w->qtnode);
        w->have_qtnode = 1;
    }
    ox_sa_boundary(g, m, p, q, w->gama, w->qt, w->vist);
    sa_viscosity(g, q, w->qt, w->visl, w->vist);
    if (p->gradient == 2) ox_gradient_ggnode(g, m, w->qt, w->qtnode, w->dntx, w->dnty, w->dntz);
    else ox_gradient(g, m, p, w->qt, w->dntx, w->dnty, w->dntz);
}

void ox_sa_residual_phase(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w)
{
    int nt = ntot(g), nc = g->n_cell;
    /* TurbSolver::UpdateResiduals (TurbSolver.cpp:316-346) */
    ox_sa_boundary(g, m, p, q, w->gama, w->qt, w->vist);
    for (int i = 0; i < nt; ++i) w->spec_t[i] = 0.0;
    for (int c = 0; c < nc; ++c) w->spec_t[c] = 0.0 * m->vol[c] + 1.0 / (p->turb_cfl_scale * w->dt[c] + OX_SMALL);
    sa_source(g, m, p, q, w);
    sa_convection(g, m, q, w);
    sa_diffusion(g, m, p, q, w);
    /* Controller::LUSGS: Diagonal */
    sa_spectrum(g, m, p, q, w);
}

void ox_sa_post_phase(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w)
{
    /* PostSolve: SetBoundaryValueOfField, then the node values of nu~ */
    ox_sa_boundary(g, m, p, q, w->gama, w->qt, w->vist);
    if (p->gradient == 2 && w->qtnode) ox_qturb_node_values(g, w->qt, w->qtnode);
}

void ox_sa_step(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, ox_ns_work *w)
{
    double *dfl = malloc(sizeof(double) * (size_t)ntot(g));
    ox_sa_gradient_phase(g, m, p, q, w);
    ox_sa_residual_phase(g, m, p, q, w);
    /* Controller::LUSGS: sweeps, UpdateFlowField */
    sa_sweep_forward(g, m, w, dfl);
    sa_sweep_backward(g, m, w, dfl);
    free(dfl);
    ox_sa_post_phase(g, m, p, q, w);
}

/* CorrectGradient, API/Physics/src/GradientOperation.cpp:21-31. */
static void correct_gradient(double fl, double fr, double *dfdx, double *dfdy, double *dfdz, double dx, double dy,
                             double dz, double ods)
{
    double fold = *dfdx * dx + *dfdy * dy + *dfdz * dz;
    double fnew = (fr - fl) * ods;
    double df = fnew - fold;
    *dfdx += df * dx;
    *dfdy += df * dy;
    *dfdz += df * dz;
}

void ox_forces(const ox_grid *g, const ox_metrics *m, const ox_params *p, const double *q, const ox_ns_work *w,
               double *out)
{
    int nt = ntot(g), nc = g->n_cell;
    double ca_f = 0, ca_p = 0, cn_f = 0, cn_p = 0, cz_f = 0, cz_p = 0, cpx = 0, cpy = 0, cpz = 0;
    double cl_f = 0, cl_p = 0, cnm_f = 0, cnm_p = 0, cm_f = 0, cm_p = 0;
    double poo = p->prim_inf[4];
    double ore = p->viscous ? 1.0 / p->reynolds : 0.0;
    /* regions in order, faces of a region in face order */
    for (int r = 0; r < g->n_region; ++r) {
        if (g->region_type[r] != OX_BC_SOLID_SURFACE) continue;
        for (int f = 0; f < g->n_bface; ++f) {
            if (g->bface_region[f] != r) continue;
            int le = g->left[f], re = nc + f;
            double nx = m->xfn[f] * m->area[f], ny = m->yfn[f] * m->area[f], nz = m->zfn[f] * m->area[f];
            double pw = q[4 * nt + le];
            double cp = 2.0 * (pw - poo);
            double dpx = nx * cp, dpy = ny * cp, dpz = nz * cp;
            ca_p += dpx; cn_p += dpy; cz_p += dpz;
            double xc = m->xfc[f], yc = m->yfc[f], zc = m->zfc[f];
            if (p->viscous) {
                double dudx = w->dqdx[nt + le], dudy = w->dqdy[nt + le], dudz = w->dqdz[nt + le];
                double dvdx = w->dqdx[2 * nt + le], dvdy = w->dqdy[2 * nt + le], dvdz = w->dqdz[2 * nt + le];
                double dwdx = w->dqdx[3 * nt + le], dwdy = w->dqdy[3 * nt + le], dwdz = w->dqdz[3 * nt + le];
                double dx = m->xcc[re] - m->xcc[le], dy = m->ycc[re] - m->ycc[le], dz = m->zcc[re] - m->zcc[le];
                double ods = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
                dx = dx * ods; dy = dy * ods; dz = dz * ods;
                correct_gradient(q[nt + le], q[nt + re], &dudx, &dudy, &dudz, dx, dy, dz, ods);
                correct_gradient(q[2 * nt + le], q[2 * nt + re], &dvdx, &dvdy, &dvdz, dx, dy, dz, ods);
                correct_gradient(q[3 * nt + le], q[3 * nt + re], &dwdx, &dwdy, &dwdz, dx, dy, dz, ods);
                double vis = w->visl[le];
                const double c23 = 2.0 / 3.0;
                double txx = vis * c23 * (2.0 * dudx - dvdy - dwdz);
                double tyy = vis * c23 * (2.0 * dvdy - dwdz - dudx);
                double tzz = vis * c23 * (2.0 * dwdz - dudx - dvdy);
                double txy = vis * (dudy + dvdx), txz = vis * (dudz + dwdx), tyz = vis * (dvdz + dwdy);
                double fvsx = -2.0 * (nx * txx + ny * txy + nz * txz) * ore;
                double fvsy = -2.0 * (nx * txy + ny * tyy + nz * tyz) * ore;
                double fvsz = -2.0 * (nx * txz + ny * tyz + nz * tzz) * ore;
                ca_f += fvsx; cn_f += fvsy; cz_f += fvsz;
                cl_f += yc * fvsz - zc * fvsy;
                cnm_f += zc * fvsx - xc * fvsz;
                cm_f += xc * fvsy - yc * fvsx;
            }
            cl_p += yc * dpz - zc * dpy;
            cnm_p += zc * dpx - xc * dpz;
            cm_p += xc * dpy - yc * dpx;
            cpx += dpx; cpy += dpy; cpz += dpz;
        }
    }
    double v[16] = {ca_f, ca_p, cn_f, cn_p, cz_f, cz_p, cpx, cpy, cpz, cl_f, cl_p, cnm_f, cnm_p, cm_f, cm_p, 0.0};
    for (int k = 0; k < 16; ++k) out[k] = v[k];
}
