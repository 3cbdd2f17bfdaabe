// Host I/O of the reference's text formats (the drop-in boundary's files).
//
// dem.data is read line by line with the same sscanf patterns as
// readDataFile (source/DEM-MPH.cpp:621-679): the patterns ARE the format, so
// they are kept identical; '#' lines are comments and any other unmatched line
// is reported and ignored.  .grid/.prof follow readGridFile (:681-851) and
// writeProfFile (:853-877).
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/dmph.h"

namespace {
thread_local std::string g_io_msg;

struct Arr6 {
    const char *fmt;
    size_t off;
};
}  // namespace

extern "C" void dmph_params_default(dmph_params *p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->dim = 3;
    p->dt = 1.0e100;
    p->dem_dt = 1.0e100;
}

extern "C" const char *dmph_io_last_message(void) { return g_io_msg.c_str(); }

#define D6(f) &p->f[0], &p->f[1], &p->f[2], &p->f[3], &p->f[4], &p->f[5]

extern "C" int dmph_read_data_file(const char *path, dmph_params *p)
{
    g_io_msg.clear();
    if (!path || !p) return DMPH_EINVAL;
    FILE *fp = std::fopen(path, "r");
    if (!fp) {
        g_io_msg = std::string("cannot open ") + path;
        return DMPH_EIO;
    }
    char buf[1024];
    while (!std::feof(fp) && !std::ferror(fp)) {
        if (std::fgets(buf, sizeof(buf), fp) == NULL) continue;
        if (buf[0] == '#') continue;
        double(*ir)[6] = p->interaction_ratio;
        if (std::sscanf(buf, " Dt %lf", &p->dt) == 1) {
        } else if (std::sscanf(buf, " DEMDt %lf", &p->dem_dt) == 1) {
        } else if (std::sscanf(buf, " OutputInterval %lf", &p->output_interval) == 1) {
        } else if (std::sscanf(buf, " VtkOutputInterval %lf", &p->vtk_output_interval) == 1) {
        } else if (std::sscanf(buf, " EndTime %lf", &p->end_time) == 1) {
        } else if (std::sscanf(buf, " RadiusRatioA %lf", &p->radius_ratio_a) == 1) {
        } else if (std::sscanf(buf, " RadiusRatioP %lf", &p->radius_ratio_p) == 1) {
        } else if (std::sscanf(buf, " RadiusRatioV %lf", &p->radius_ratio_v) == 1) {
        } else if (std::sscanf(buf, " Density %lf %lf %lf %lf %lf %lf", D6(density)) == 6) {
        } else if (std::sscanf(buf, " BulkModulus %lf %lf %lf %lf %lf %lf", D6(bulk_modulus)) == 6) {
        } else if (std::sscanf(buf, " BulkViscosity %lf %lf %lf %lf %lf %lf", D6(bulk_viscosity)) == 6) {
        } else if (std::sscanf(buf, " ShearViscosity %lf %lf %lf %lf %lf %lf", D6(shear_viscosity)) == 6) {
        } else if (std::sscanf(buf, " SurfaceTension %lf %lf %lf %lf %lf %lf", D6(surface_tension)) == 6) {
        } else if (std::sscanf(buf, " InteractionRatio(Type0) %lf %lf %lf %lf %lf %lf", &ir[0][0], &ir[0][1],
                               &ir[0][2], &ir[0][3], &ir[0][4], &ir[0][5]) == 6) {
        } else if (std::sscanf(buf, " InteractionRatio(Type1) %lf %lf %lf %lf %lf %lf", &ir[1][0], &ir[1][1],
                               &ir[1][2], &ir[1][3], &ir[1][4], &ir[1][5]) == 6) {
        } else if (std::sscanf(buf, " InteractionRatio(Type2) %lf %lf %lf %lf %lf %lf", &ir[2][0], &ir[2][1],
                               &ir[2][2], &ir[2][3], &ir[2][4], &ir[2][5]) == 6) {
        } else if (std::sscanf(buf, " InteractionRatio(Type3) %lf %lf %lf %lf %lf %lf", &ir[3][0], &ir[3][1],
                               &ir[3][2], &ir[3][3], &ir[3][4], &ir[3][5]) == 6) {
        } else if (std::sscanf(buf, " InteractionRatio(Type4) %lf %lf %lf %lf %lf %lf", &ir[4][0], &ir[4][1],
                               &ir[4][2], &ir[4][3], &ir[4][4], &ir[4][5]) == 6) {
        } else if (std::sscanf(buf, " InteractionRatio(Type5) %lf %lf %lf %lf %lf %lf", &ir[5][0], &ir[5][1],
                               &ir[5][2], &ir[5][3], &ir[5][4], &ir[5][5]) == 6) {
        } else if (std::sscanf(buf, " Gravity %lf %lf %lf", &p->gravity[0], &p->gravity[1], &p->gravity[2]) == 3) {
        } else if (std::sscanf(buf, " YoungModulus %lf %lf %lf %lf %lf %lf   ", D6(young_modulus)) == 6) {
        } else if (std::sscanf(buf, " PoissonRatio %lf %lf %lf %lf %lf %lf ", D6(poisson_ratio)) == 6) {
        } else if (std::sscanf(buf, " RestitutionCoefficient  %lf %lf %lf %lf %lf %lf ",
                               D6(restitution_coefficient)) == 6) {
        } else if (std::sscanf(buf, " ViscousFrictionCoefficient %lf %lf %lf %lf %lf %lf ",
                               D6(viscous_friction_coefficient)) == 6) {
        } else if (std::sscanf(buf, " Wall4  Center %lf %lf %lf Velocity %lf %lf %lf Omega %lf %lf %lf",
                               &p->wall_center[4][0], &p->wall_center[4][1], &p->wall_center[4][2],
                               &p->wall_velocity[4][0], &p->wall_velocity[4][1], &p->wall_velocity[4][2],
                               &p->wall_omega[4][0], &p->wall_omega[4][1], &p->wall_omega[4][2]) == 9) {
        } else if (std::sscanf(buf, " Wall5  Center %lf %lf %lf Velocity %lf %lf %lf Omega %lf %lf %lf",
                               &p->wall_center[5][0], &p->wall_center[5][1], &p->wall_center[5][2],
                               &p->wall_velocity[5][0], &p->wall_velocity[5][1], &p->wall_velocity[5][2],
                               &p->wall_omega[5][0], &p->wall_omega[5][1], &p->wall_omega[5][2]) == 9) {
        } else {
            g_io_msg += "Invalid line in data file \"";
            g_io_msg += buf;
            g_io_msg += "\"\n";
        }
    }
    std::fclose(fp);
    return DMPH_OK;
}

extern "C" int dmph_read_grid_file(const char *path, dmph_params *p, int *n, int *type, double *x3, double *v3)
{
    g_io_msg.clear();
    if (!path || !p || !n) return DMPH_EINVAL;
    FILE *fp = std::fopen(path, "r");
    if (!fp) {
        g_io_msg = std::string("cannot open ") + path;
        return DMPH_EIO;
    }
    char buf[1024];
    int count = 0;
    double t = 0.0, dx = 0.0, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    if (std::fgets(buf, sizeof(buf), fp) == NULL || std::sscanf(buf, "%lf", &t) != 1 ||
        std::fgets(buf, sizeof(buf), fp) == NULL ||
        std::sscanf(buf, "%d  %lf  %lf %lf %lf  %lf %lf %lf", &count, &dx, &lo[0], &hi[0], &lo[1], &hi[1], &lo[2],
                    &hi[2]) != 8 ||
        count <= 0) {
        std::fclose(fp);
        g_io_msg = std::string("bad grid header in ") + path;
        return DMPH_EIO;
    }
    p->time = t;
    p->particle_spacing = dx;
    for (int d = 0; d < 3; d++) {
        p->domain_min[d] = lo[d];
        p->domain_max[d] = hi[d];
    }
    if (!type) {
        *n = count;
        std::fclose(fp);
        return DMPH_OK;
    }
    if (*n < count || !x3 || !v3) {
        std::fclose(fp);
        return DMPH_EINVAL;
    }
    int i = 0;
    for (; i < count; ++i) {
        if (std::fgets(buf, sizeof(buf), fp) == NULL) break;
        if (std::sscanf(buf, "%d  %lf %lf %lf  %lf %lf %lf", &type[i], &x3[3 * i], &x3[3 * i + 1], &x3[3 * i + 2],
                        &v3[3 * i], &v3[3 * i + 1], &v3[3 * i + 2]) != 7)
            break;
        if (type[i] < 0 || type[i] >= DMPH_TYPE_COUNT) break;
    }
    std::fclose(fp);
    if (i != count) {
        g_io_msg = std::string("grid ") + path + ": bad or missing particle row " + std::to_string(i);
        return DMPH_EIO;
    }
    *n = count;
    return DMPH_OK;
}

extern "C" int dmph_write_prof_file(const char *path, const dmph_params *p, int n, const int *type, const double *x3,
                                    const double *v3)
{
    if (!path || !p || n < 0 || (n > 0 && (!type || !x3 || !v3))) return DMPH_EINVAL;
    FILE *fp = std::fopen(path, "w");
    if (!fp) {
        g_io_msg = std::string("cannot write ") + path;
        return DMPH_EIO;
    }
    std::fprintf(fp, "%e\n", p->time);
    std::fprintf(fp, "%d %e %e %e %e %e %e %e\n", n, p->particle_spacing, p->domain_min[0], p->domain_max[0],
                 p->domain_min[1], p->domain_max[1], p->domain_min[2], p->domain_max[2]);
    for (int i = 0; i < n; ++i)
        std::fprintf(fp, "%d %e %e %e  %e %e %e\n", type[i], x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], v3[3 * i],
                     v3[3 * i + 1], v3[3 * i + 2]);
    std::fflush(fp);
    const int bad = std::ferror(fp);
    std::fclose(fp);
    return bad ? DMPH_EIO : DMPH_OK;
}

// The VTK output of writeVtkFile (source/DEM-MPH.cpp:879-1005): legacy ASCII
// unstructured grid of vertices with the reference's point data, in its order
// and with its number formats (positions and velocities rounded to float).
extern "C" int dmph_write_vtk_file(const char *path, int n, const int *type, const double *x3, const double *v3,
                                   const double *kn, const double *cn, const double *kt, const double *ct,
                                   const int *neighbor_count, const double *alpha, const double *drag,
                                   const double *vol_strain, const double *virial_pressure)
{
    if (!path || n < 0) return DMPH_EINVAL;
    if (n > 0 && (!type || !x3 || !v3 || !kn || !cn || !kt || !ct || !neighbor_count || !alpha || !drag ||
                  !vol_strain || !virial_pressure))
        return DMPH_EINVAL;
    FILE *fp = std::fopen(path, "w");
    if (!fp) {
        g_io_msg = std::string("cannot write ") + path;
        return DMPH_EIO;
    }
    std::fprintf(fp, "# vtk DataFile Version 2.0\n");
    std::fprintf(fp, "Unstructured Grid Example\n");
    std::fprintf(fp, "ASCII\n");
    std::fprintf(fp, "DATASET UNSTRUCTURED_GRID\n");
    std::fprintf(fp, "POINTS %d float\n", n);
    for (int i = 0; i < n; ++i)
        std::fprintf(fp, "%e %e %e\n", (float)x3[3 * i], (float)x3[3 * i + 1], (float)x3[3 * i + 2]);
    std::fprintf(fp, "CELLS %d %d\n", n, 2 * n);
    for (int i = 0; i < n; ++i) std::fprintf(fp, "1 %d ", i);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "CELL_TYPES %d\n", n);
    for (int i = 0; i < n; ++i) std::fprintf(fp, "1 ");
    std::fprintf(fp, "\n");
    std::fprintf(fp, "\n");
    std::fprintf(fp, "POINT_DATA %d\n", n);
    std::fprintf(fp, "SCALARS label float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%d\n", type[i]);
    std::fprintf(fp, "\n");
    const struct {
        const char *name;
        const double *a;
    } dem[4] = {{"NormalSpringConstant", kn},
                {"NormalViscousDampingConstant", cn},
                {"TangentialSpringConstant", kt},
                {"TangentialViscousDampingConstant", ct}};
    for (const auto &f : dem) {
        std::fprintf(fp, "SCALARS %s float 1\n", f.name);
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (int i = 0; i < n; ++i) std::fprintf(fp, "%e\n", f.a[i]);
    }
    std::fprintf(fp, "SCALARS neighbor float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%d\n", neighbor_count[i]);
    std::fprintf(fp, "SCALARS volumef float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%e\n", alpha[i]);
    std::fprintf(fp, "SCALARS drag float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%e\n", drag[i]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "VECTORS velocity float\n");
    for (int i = 0; i < n; ++i)
        std::fprintf(fp, "%e %e %e\n", (float)v3[3 * i], (float)v3[3 * i + 1], (float)v3[3 * i + 2]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "SCALARS VolStrainP float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%e\n", (float)vol_strain[i]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "SCALARS VirialPressureAtParticle float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%e\n", (float)virial_pressure[i]);
    std::fprintf(fp, "\n");
    std::fflush(fp);
    const int bad = std::ferror(fp);
    std::fclose(fp);
    return bad ? DMPH_EIO : DMPH_OK;
}
