// The reference's host-side membrane pieces, compiled from its own sources:
// the ring adjacency (src/rbc/adj/imp.cpp: adj_ini, the host adj_get_map,
// src/algo/edg) and the host build of the Kantor dihedral forces
// (src/mesh/force/kantor0/imp.cpp, FORCE_KANTOR0_HOST: FP64, pow(x, -0.5) for
// rsqrt).  This file supplies what those sources take from modules that need
// a GPU or a log: the device-memory calls of adj_view_ini (never called here:
// the tests copy the tables to the device themselves), the CUDA check and a
// no-op log.
// TEST INFRASTRUCTURE ONLY: only tests/ load the resulting library.
#include <stdio.h>
#include <stdlib.h>
#include <math.h>
#include <vector_types.h>

#include "utils/error.h"
#include "math/dev.h"
#include "rbc/adj/imp.h"
#include "rbc/adj/type/common.h"
#include "rbc/adj/imp/type.h"
#include "mesh/force/kantor0/imp.h"

namespace d {
int Malloc(void **, size_t) { fprintf(stderr, "refhost: no device memory here\n"); abort(); }
int Memcpy(void *, const void *, size_t, int) { fprintf(stderr, "refhost: no device memory here\n"); abort(); }
int Free(void *) { fprintf(stderr, "refhost: no device memory here\n"); abort(); }
}
namespace cc {
void check(int rc, const char *file, int line) {
    if (rc) { fprintf(stderr, "refhost: %s:%d: code %d\n", file, line, rc); abort(); }
}
}
void msg_print(const char *, ...) {}

/* adj_ini (src/rbc/adj/imp/ini.h:34-45): adj0, adj1 [md nv] of the template
 * of nt triangles tri4 (int4 a triangle) */
extern "C" int refhost_adj(int md, int nt, int nv, const int *tri4, int *adj0, int *adj1) {
    Adj *q;
    adj_ini(md, nt, nv, (const int4 *)tri4, &q);
    for (int i = 0; i < md * nv; i++) { adj0[i] = q->adj0[i]; adj1[i] = q->adj1[i]; }
    adj_fin(q);
    return 0;
}

/* the Kantor forces of nc cells of nv vertices pp [AoS, 6 floats] added to ff
 * [3 doubles a vertex]: the traversal of kantor_dev::force
 * (src/rbc/force/bending/kantor/dev/main.h:23-66) on the host, each (vertex,
 * ring slot) through the host adj_get_map, with the host dih_a / dih_b */
extern "C" int refhost_kantor(double phi_deg, double kb, int md, int nt, int nv, const int *tri4, int nc,
                              const float *pp, double *ff) {
    Adj *q;
    adj_ini(md, nt, nv, (const int4 *)tri4, &q);
    const double phi = phi_deg / 180.0 * M_PI;
    for (int c = 0; c < nc; c++) {
        const int off = c * nv;
        for (int i = 0; i < md * nv; i++) {
            AdjMap m;
            if (!adj_get_map(i, q, &m)) continue;
            double3 r[5];
            const int id[5] = {m.i0, m.i1, m.i2, m.i3, m.i4};
            for (int j = 0; j < 5; j++) {
                const float *p = pp + 6 * (size_t)(off + id[j]);
                r[j].x = p[0]; r[j].y = p[1]; r[j].z = p[2];
            }
            const double3 fa = force_kantor0_hst::dih_a(phi, kb, r[0], r[2], r[1], r[4]);
            const double3 fb = force_kantor0_hst::dih_b(phi, kb, r[1], r[0], r[2], r[3]);
            double *f = ff + 3 * (size_t)(off + m.i0);
            f[0] += fa.x + fb.x; f[1] += fa.y + fb.y; f[2] += fa.z + fb.z;
        }
    }
    adj_fin(q);
    return 0;
}
