// Membrane mesh dumps in the reference's PLY format (host code).
//
// mesh_write_particles (src/io/mesh/imp/main.h:52-134) of one rank: the
// header text of its header(), then nc * nv vertices as six little-endian
// floats (x, y, z, u, v, w), then nc * nt faces as four little-endian ints
// (3, i0, i1, i2) with the vertex indices of cell c shifted by c * nv.
// Positions go through the reference's transform of its shift type
// (src/algo/vectors/imp/main.h:15-54 with src/math/tform): for one rank the
// edge origin is x + L/2 (scale 1, origin L/2, in float) and the centre
// origin leaves x as it is.
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/ctc_b200.h"
#include "api_util.h"

extern "C" int ctc_mesh_write_ply(const char *path, int nc, int nv, int nt, const int *tri, const float *pp, int shift,
                                  int LX, int LY, int LZ) {
    using ctc::fail;
    if (!path || nc < 0 || nv <= 0 || nt <= 0 || !tri || (nc > 0 && !pp) || (shift != 0 && shift != 1))
        return fail(CTC_ERR_ARG, "ctc_mesh_write_ply: bad arguments");
    for (int k = 0; k < 3 * nt; k++)
        if (tri[k] < 0 || tri[k] >= nv) return fail(CTC_ERR_ARG, "ctc_mesh_write_ply: bad triangle %d", k / 3);
    FILE *f = fopen(path, "wb");
    if (!f) return fail(CTC_ERR_ARG, "ctc_mesh_write_ply: cannot open %s", path);
    char head[1024];
    const int hs = snprintf(head, sizeof(head),
                            "ply\n"
                            "format binary_little_endian 1.0\n"
                            "element vertex %d\n"
                            "property float x\nproperty float y\nproperty float z\n"
                            "property float u\nproperty float v\nproperty float w\n"
                            "element face  %d\n"
                            "property list int int vertex_index\n"
                            "end_header\n",
                            nv * nc, nt * nc);
    bool ok = fwrite(head, 1, (size_t)hs, f) == (size_t)hs;
    const float o[3] = {shift == 0 ? 0.5f * (float)LX : 0.0f, shift == 0 ? 0.5f * (float)LY : 0.0f,
                        shift == 0 ? 0.5f * (float)LZ : 0.0f};
    std::vector<float> v(6 * (size_t)nv * nc);
    for (size_t i = 0; i < (size_t)nv * nc; i++) {
        for (int k = 0; k < 3; k++) v[6 * i + k] = pp[6 * i + k] + o[k];   // s x + o with s = 1
        for (int k = 3; k < 6; k++) v[6 * i + k] = pp[6 * i + k];
    }
    ok = ok && fwrite(v.data(), sizeof(float), v.size(), f) == v.size();
    std::vector<int> fa(4 * (size_t)nt * nc);
    for (int c = 0; c < nc; c++)
        for (int t = 0; t < nt; t++) {
            int *q = fa.data() + 4 * ((size_t)c * nt + t);
            q[0] = 3;
            for (int k = 0; k < 3; k++) q[1 + k] = nv * c + tri[3 * t + k];
        }
    ok = ok && fwrite(fa.data(), sizeof(int), fa.size(), f) == fa.size();
    ok = (fclose(f) == 0) && ok;
    return ok ? CTC_OK : fail(CTC_ERR_ARG, "ctc_mesh_write_ply: write failed on %s", path);
}
