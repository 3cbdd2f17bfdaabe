// Rigid debris bodies at the drop-in boundary: the body sidecar file and the
// membership by contact.
//
// The reference's .grid rows carry a type and a state only
// (generator/generator.cpp:97, 211-214; readGridFile source/DEM-MPH.cpp:
// 681-851), and its two solid types are its only densities, so a scene of
// rigid debris bodies with their own densities needs a second file beside
// the .grid.  Its format (text, one value per line after a header):
//
//     DMPH_BODIES 1
//     <nbodies> <nrows>
//     <density of body 0>            nbodies lines, kg/m^3
//     ...
//     <body of grid row 0>           nrows lines, -1 for no body
//     ...
//
// Without a sidecar, bodies are the connected components of the solid
// particles under contact at 1.01 dx (two solid particles closer than
// 1.01 ParticleSpacing, periodic minimum image, belong to one body), each with
// the density of its first row's type: the debris blocks of a generator
// lattice sit at dx spacing, so every block is one component unless two
// blocks touch.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/dmph.h"

namespace {

thread_local std::string g_bodies_msg;

int io_fail(int code, const std::string &m)
{
    g_bodies_msg = m;
    return code;
}

bool is_solid_type(int t) { return DMPH_SOLID_BEGIN <= t && t < DMPH_SOLID_END; }

// union-find over solid rows, roots the smallest row of each component
struct Dsu {
    std::vector<int> up;
    explicit Dsu(int n) : up(n) { std::iota(up.begin(), up.end(), 0); }
    int find(int a)
    {
        while (up[a] != a) {
            up[a] = up[up[a]];
            a = up[a];
        }
        return a;
    }
    void join(int a, int b)
    {
        a = find(a);
        b = find(b);
        if (a == b) return;
        if (b < a) std::swap(a, b);
        up[b] = a;
    }
};

}  // namespace

extern "C" const char *dmph_bodies_last_message(void) { return g_bodies_msg.c_str(); }

extern "C" int dmph_write_bodies_file(const char *path, int nbodies, int nrows, const int *body_of_row,
                                      const double *body_density)
{
    g_bodies_msg.clear();
    if (!path || nbodies < 0 || nrows < 0 || (nrows && !body_of_row) || (nbodies && !body_density))
        return io_fail(DMPH_EINVAL, "null argument or negative size");
    FILE *fp = std::fopen(path, "w");
    if (!fp) return io_fail(DMPH_EIO, std::string("cannot open ") + path);
    std::fprintf(fp, "DMPH_BODIES 1\n%d %d\n", nbodies, nrows);
    for (int b = 0; b < nbodies; b++) std::fprintf(fp, "%.17g\n", body_density[b]);
    for (int r = 0; r < nrows; r++) std::fprintf(fp, "%d\n", body_of_row[r]);
    const bool ok = !std::ferror(fp);
    std::fclose(fp);
    return ok ? DMPH_OK : io_fail(DMPH_EIO, std::string("cannot write ") + path);
}

extern "C" int dmph_read_bodies_file(const char *path, int *nbodies, int *nrows, int *body_of_row,
                                     double *body_density)
{
    g_bodies_msg.clear();
    if (!path || !nbodies || !nrows) return io_fail(DMPH_EINVAL, "null argument");
    FILE *fp = std::fopen(path, "r");
    if (!fp) return io_fail(DMPH_EIO, std::string("cannot open ") + path);
    int version = 0, B = -1, R = -1;
    int rc = DMPH_OK;
    if (std::fscanf(fp, " DMPH_BODIES %d", &version) != 1 || version != 1)
        rc = io_fail(DMPH_EIO, std::string(path) + ": not a DMPH_BODIES 1 file");
    else if (std::fscanf(fp, "%d %d", &B, &R) != 2 || B < 0 || R < 0)
        rc = io_fail(DMPH_EIO, std::string(path) + ": bad body or row count");
    if (!rc && (body_of_row || body_density)) {
        if (!body_of_row || !body_density || *nbodies < B || *nrows < R)
            rc = io_fail(DMPH_ERANGE, "arrays smaller than the file's counts");
        for (int b = 0; !rc && b < B; b++)
            if (std::fscanf(fp, "%lf", &body_density[b]) != 1 || !(body_density[b] > 0.0))
                rc = io_fail(DMPH_EIO, std::string(path) + ": bad density of body " + std::to_string(b));
        for (int r = 0; !rc && r < R; r++)
            if (std::fscanf(fp, "%d", &body_of_row[r]) != 1 || body_of_row[r] < -1 || body_of_row[r] >= B)
                rc = io_fail(DMPH_EIO, std::string(path) + ": bad body of row " + std::to_string(r));
    }
    std::fclose(fp);
    if (!rc) {
        *nbodies = B;
        *nrows = R;
    }
    return rc;
}

extern "C" int dmph_bodies_from_contacts(const dmph_params *p, int n, const int *type, const double *x3,
                                         int *body_of_row, int *nbodies, double *body_density, int density_capacity)
{
    g_bodies_msg.clear();
    if (!p || n <= 0 || !type || !x3 || !body_of_row || !nbodies) return io_fail(DMPH_EINVAL, "null argument");
    const int dim = p->dim == 2 ? 2 : 3;
    const double reach = 1.01 * p->particle_spacing;
    if (!(reach > 0.0)) return io_fail(DMPH_EINVAL, "ParticleSpacing must be positive");
    double W[3], cw[3];
    int nc[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) {
        W[d] = p->domain_max[d] - p->domain_min[d];
        if (!(W[d] > 0.0)) return io_fail(DMPH_EINVAL, "empty domain extent");
        nc[d] = std::max(1, (int)std::floor(W[d] / reach));
        nc[d] = std::min(nc[d], 1 << 20);
        cw[d] = W[d] / nc[d];
    }
    std::vector<int> solids;
    for (int r = 0; r < n; r++) {
        body_of_row[r] = -1;
        if (is_solid_type(type[r])) solids.push_back(r);
    }
    const int S = (int)solids.size();
    // bin the solids by cell (a sort by cell key), then test the 3^dim
    // neighbouring cells of each
    auto cell_of = [&](int r, int c[3]) {
        for (int d = 0; d < 3; d++) c[d] = 0;
        for (int d = 0; d < dim; d++) {
            const double u = (x3[3 * (size_t)r + d] - p->domain_min[d]) / cw[d];
            long long k = (long long)std::floor(u);
            k %= nc[d];
            if (k < 0) k += nc[d];
            c[d] = (int)k;
        }
    };
    auto key_of = [&](const int c[3]) { return ((long long)c[0] * nc[1] + c[1]) * nc[2] + c[2]; };
    std::vector<std::pair<long long, int>> keyed(S);
    for (int s = 0; s < S; s++) {
        int c[3];
        cell_of(solids[s], c);
        keyed[s] = {key_of(c), s};
    }
    std::sort(keyed.begin(), keyed.end());
    std::vector<long long> keys(S);
    for (int s = 0; s < S; s++) keys[s] = keyed[s].first;
    Dsu dsu(S);
    const double reach2 = reach * reach;
    for (int s = 0; s < S; s++) {
        const int r = solids[s];
        int c[3];
        cell_of(r, c);
        long long seen[27];
        int nseen = 0;
        const int zr = dim == 3 ? 1 : 0;
        for (int ox = -1; ox <= 1; ox++)
            for (int oy = -1; oy <= 1; oy++)
                for (int oz = -zr; oz <= zr; oz++) {
                    int cc[3] = {((c[0] + ox) % nc[0] + nc[0]) % nc[0], ((c[1] + oy) % nc[1] + nc[1]) % nc[1],
                                 ((c[2] + oz) % nc[2] + nc[2]) % nc[2]};
                    const long long k = key_of(cc);
                    if (std::find(seen, seen + nseen, k) != seen + nseen) continue;  // axes of < 3 cells
                    seen[nseen++] = k;
                    auto lo = std::lower_bound(keys.begin(), keys.end(), k);
                    for (auto it = lo; it != keys.end() && *it == k; ++it) {
                        const int t = keyed[it - keys.begin()].second;
                        if (t <= s) continue;  // each pair once
                        const int q = solids[t];
                        double d2 = 0.0;
                        for (int d = 0; d < dim; d++) {
                            double a = x3[3 * (size_t)q + d] - x3[3 * (size_t)r + d];
                            a -= W[d] * std::floor(a / W[d] + 0.5);  // minimum image
                            d2 += a * a;
                        }
                        if (d2 <= reach2) dsu.join(s, t);
                    }
                }
    }
    // bodies numbered by their first row, in row order
    std::vector<int> body_of_root(S, -1);
    int B = 0;
    for (int s = 0; s < S; s++) {  // solids are in row order
        const int root = dsu.find(s);
        if (body_of_root[root] < 0) body_of_root[root] = B++;
        body_of_row[solids[s]] = body_of_root[root];
    }
    *nbodies = B;
    if (body_density) {
        if (density_capacity < B) return io_fail(DMPH_ERANGE, "body_density holds fewer than the bodies found");
        std::vector<char> set(B, 0);
        for (int s = 0; s < S; s++) {
            const int b = body_of_row[solids[s]];
            if (!set[b]) {
                body_density[b] = p->density[type[solids[s]]];
                set[b] = 1;
            }
        }
    }
    return DMPH_OK;
}
