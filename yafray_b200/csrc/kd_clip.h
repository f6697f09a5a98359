// Triangle-against-box clipping of the kd build, for host and device.
//
// Sutherland-Hodgman clip of a triangle against an axis-aligned box in
// double (triBoxClip, triclip.cc:50-240): the three axes in order, the
// lower plane before the upper one, a vertex on a plane counted as inside.
// The kd build bounds the clipped polygon to get a triangle's extent
// inside a node of at most 32 triangles (kdtree.cc:430-470).
#pragma once

#include "kd_sort.h"  // YR_HD

namespace yr {

// Returns 0 with the clipped bound in (lo, hi), 1 when nothing is left,
// 2 when the polygon outgrows its buffer (the caller keeps the full bound).
YR_HD int kd_clip_triangle(const double bmin[3], const double bmax[3], const double v[3][3], float lo[3],
                           float hi[3]) {
    double buf1[11][3], buf2[11][3];
    double(*poly)[3] = buf1;
    double(*cpoly)[3] = buf2;
    for (int q = 0; q < 3; q++) {
        poly[q][0] = v[q][0];
        poly[q][1] = v[q][1];
        poly[q][2] = v[q][2];
        poly[3][q] = v[0][q];
    }
    int n = 3;
    for (int axis = 0; axis < 3; axis++) {
        const int na = (axis + 1) % 3, pa = (axis + 2) % 3;
        for (int side = 0; side < 2; side++) {
            // side 0 clips against the lower plane, side 1 against the upper one
            const double plane = side == 0 ? bmin[axis] : bmax[axis];
            int nc = 0;
            bool p1_in = side == 0 ? (poly[0][axis] >= plane) : (poly[0][axis] <= plane);
            for (int i = 0; i < n; i++) {
                const double *p1 = poly[i], *p2 = poly[i + 1];
                const bool p2_in = side == 0 ? (p2[axis] >= plane) : (p2[axis] <= plane);
                const bool p2_strict = side == 0 ? (p2[axis] > plane) : (p2[axis] < plane);
                if (p1_in) {
                    if (p2_in) {
                        for (int k = 0; k < 3; k++) cpoly[nc][k] = p2[k];
                        nc++;
                        p1_in = true;
                    } else {
                        const double t = (plane - p1[axis]) / (p2[axis] - p1[axis]);
                        cpoly[nc][axis] = plane;
                        cpoly[nc][na] = p1[na] + t * (p2[na] - p1[na]);
                        cpoly[nc][pa] = p1[pa] + t * (p2[pa] - p1[pa]);
                        nc++;
                        p1_in = false;
                    }
                } else {
                    if (p2_strict) {
                        const double t = (plane - p2[axis]) / (p1[axis] - p2[axis]);
                        cpoly[nc][axis] = plane;
                        cpoly[nc][na] = p2[na] + t * (p1[na] - p2[na]);
                        cpoly[nc][pa] = p2[pa] + t * (p1[pa] - p2[pa]);
                        nc++;
                        for (int k = 0; k < 3; k++) cpoly[nc][k] = p2[k];
                        nc++;
                        p1_in = true;
                    } else if (p2[axis] == plane) {
                        for (int k = 0; k < 3; k++) cpoly[nc][k] = p2[k];
                        nc++;
                        p1_in = true;
                    } else {
                        p1_in = false;
                    }
                }
            }
            if (nc > 9) return 2;
            for (int k = 0; k < 3; k++) cpoly[nc][k] = cpoly[0][k];
            n = nc;
            double(*tmp)[3] = poly;
            poly = cpoly;
            cpoly = tmp;
        }
    }
    if (n < 2) return 1;
    double a[3], g[3];
    for (int k = 0; k < 3; k++) a[k] = g[k] = poly[0][k];
    for (int i = 1; i < n; i++)
        for (int k = 0; k < 3; k++) {
            a[k] = (poly[i][k] < a[k]) ? poly[i][k] : a[k];  // std::min
            g[k] = (g[k] < poly[i][k]) ? poly[i][k] : g[k];  // std::max
        }
    for (int k = 0; k < 3; k++) {
        lo[k] = (float)a[k];
        hi[k] = (float)g[k];
    }
    return 0;
}

}  // namespace yr
