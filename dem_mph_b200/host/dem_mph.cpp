// dem_mph — drop-in replacement of the reference solver executable.
//
//   dem_mph [--dim 2|3] [--fp32] [--gpu N] [--bodies FILE | --rigid]
//           [--checkpoint] [--resume FILE]
//           data grid prof_pattern vtk_pattern log
//
// --checkpoint writes, beside every .prof file, NAME.prof.ckpt: a checkpoint
// of the solver (dmph_checkpoint_write) with this driver's output schedule.
// --resume FILE continues the run such a file was taken from: the solver
// state, its parameters and the output schedule come from FILE, the data
// file gives EndTime (so a run can be extended) and the grid file is not
// read; no output.vtk is written.  The files written after a resume are
// byte-identical to those of the uninterrupted run.  The reference's own
// restart (a .prof file given as the grid) remains: it starts afresh from the
// positions and velocities of the file.
//
// --bodies FILE moves the debris as rigid bodies with the membership and
// densities of a body sidecar file (dmph_read_bodies_file); --rigid does the
// same with the bodies taken as the solid particles connected by contact at
// 1.01 dx, each with its type's density (dmph_bodies_from_contacts).  Without
// either, debris particles move individually, as in the reference.
//
// Same positional arguments, defaults and output cadence as the reference's
// main (source/DEM-MPH.cpp:350-617): it reads dem.data and the .grid file,
// writes a .prof (positions and velocities in the solver's sorted order) at
// the top of every step whose time reaches the next OutputInterval boundary
// and advances until EndTime; after initialisation it writes output.vtk, and
// at the end of every step whose time reaches the next VtkOutputInterval
// boundary it computes the virial pressure and writes a VTK file named by the
// VTK pattern, as the reference does (:426, :566-575).  All computation
// happens in libdmph.so through the C ABI of include/dmph.h.  The reference is
// compiled 2D by default (source/DEM-MPH.cpp:39); --dim 3 selects its 3D
// branches.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include <cuda_runtime_api.h>

#include "dmph.h"

static FILE *g_log = nullptr;

static void log_printf(const char *fmt, ...)
{
    va_list a, b;
    va_start(a, fmt);
    va_copy(b, a);
    if (g_log) vfprintf(g_log, fmt, a);
    vfprintf(stderr, fmt, b);
    va_end(a);
    va_end(b);
}

static int fail(const char *what, int rc, dmph_ctx *ctx)
{
    log_printf("%s failed (%d): %s\n", what, rc, dmph_last_error(ctx));
    return 1;
}

int main(int argc, char **argv)
{
    // defaults of the reference (:54-58)
    std::string logf = "sample.log", dataf = "sample.data", gridf = "sample.grid", proff = "sample%03d.prof",
                vtkf = "sample%03d.vtk";
    int dim = 2, fp32 = 0, gpu = 0, rigid = 0, checkpoint = 0;
    std::string bodiesf, resumef;
    std::vector<std::string> pos;
    for (int a = 1; a < argc; a++) {
        if (!std::strcmp(argv[a], "--dim") && a + 1 < argc)
            dim = std::atoi(argv[++a]);
        else if (!std::strcmp(argv[a], "--fp32"))
            fp32 = 1;
        else if (!std::strcmp(argv[a], "--gpu") && a + 1 < argc)
            gpu = std::atoi(argv[++a]);
        else if (!std::strcmp(argv[a], "--bodies") && a + 1 < argc)
            bodiesf = argv[++a];
        else if (!std::strcmp(argv[a], "--rigid"))
            rigid = 1;
        else if (!std::strcmp(argv[a], "--checkpoint"))
            checkpoint = 1;
        else if (!std::strcmp(argv[a], "--resume") && a + 1 < argc)
            resumef = argv[++a];
        else
            pos.push_back(argv[a]);
    }
    if (pos.size() > 0) dataf = pos[0];
    if (pos.size() > 1) gridf = pos[1];
    if (pos.size() > 2) proff = pos[2];
    if (pos.size() > 3) vtkf = pos[3];
    if (pos.size() > 4) logf = pos[4];
    g_log = std::fopen(logf.c_str(), "w");
    if (!g_log) std::fprintf(stderr, "error in open %s\n", logf.c_str());
    {
        time_t t = time(NULL);
        log_printf("start reading files at %s\n", ctime(&t));
    }
    dmph_params p;
    dmph_params_default(&p);
    int rc = dmph_read_data_file(dataf.c_str(), &p);
    if (rc) return log_printf("cannot read %s: %s\n", dataf.c_str(), dmph_io_last_message()), 1;
    if (*dmph_io_last_message()) log_printf("%s", dmph_io_last_message());
    if (cudaSetDevice(gpu) != cudaSuccess) return log_printf("cannot select GPU %d\n", gpu), 1;
    // this driver's part of a checkpoint: its clock and output schedule
    struct Schedule {
        double time, output_next, vtk_output_next;
        int step;
    } sched = {p.time, 0.0, 0.0, 0};
    dmph_ctx *ctx = nullptr;
    int n = 0;
    if (!resumef.empty()) {
        int nu = 0;
        rc = dmph_checkpoint_open(resumef.c_str(), &ctx, &sched, (int)sizeof(sched), &nu);
        if (rc) return fail("dmph_checkpoint_open", rc, nullptr);
        if (nu != (int)sizeof(sched)) return log_printf("%s was not written by dem_mph\n", resumef.c_str()), 1;
        const double end_time = p.end_time;
        dmph_get_params(ctx, &p);
        p.end_time = end_time;
        dmph_info inf;
        dmph_get_info(ctx, &inf);
        n = inf.n;
        log_printf("resumed from %s at Time %e (step %d)\n", resumef.c_str(), sched.time, sched.step);
    }
    if (!ctx) rc = dmph_read_grid_file(gridf.c_str(), &p, &n, nullptr, nullptr, nullptr);
    if (rc) return log_printf("cannot read %s: %s\n", gridf.c_str(), dmph_io_last_message()), 1;
    std::vector<int> type(n);
    std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n);
    if (!ctx) {
        rc = dmph_read_grid_file(gridf.c_str(), &p, &n, type.data(), x.data(), v.data());
        if (rc) return log_printf("cannot read %s: %s\n", gridf.c_str(), dmph_io_last_message()), 1;
        p.dim = dim;
        p.precision = fp32 ? DMPH_PRECISION_FP32_SPLIT : DMPH_PRECISION_FP64;
        // the VTK output carries every particle's NeighborCount and the DEM
        // constants the reference also evaluates for wall particles
        p.flags |= DMPH_FLAG_ALL_NEIGHBOR_COUNTS | DMPH_FLAG_WALL_DEM_COEFFS;
        sched.time = p.time;
    }
    {
        time_t t = time(NULL);
        log_printf("start initialization at %s\n", ctime(&t));
    }
    // rigid debris bodies: membership and densities by grid row
    std::vector<int> body_of_row;
    std::vector<double> body_density;
    int nbodies = 0;
    if (ctx) {
        // resumed: the bodies come with the checkpoint
    } else if (!bodiesf.empty()) {
        int nrows = 0;
        rc = dmph_read_bodies_file(bodiesf.c_str(), &nbodies, &nrows, nullptr, nullptr);
        if (!rc && nrows != n) return log_printf("%s has %d rows, the grid %d\n", bodiesf.c_str(), nrows, n), 1;
        body_of_row.resize(n);
        body_density.resize(nbodies > 0 ? nbodies : 1);
        if (!rc) rc = dmph_read_bodies_file(bodiesf.c_str(), &nbodies, &nrows, body_of_row.data(), body_density.data());
        if (rc) return log_printf("cannot read %s: %s\n", bodiesf.c_str(), dmph_bodies_last_message()), 1;
    } else if (rigid) {
        body_of_row.resize(n);
        body_density.resize(n);
        rc = dmph_bodies_from_contacts(&p, n, type.data(), x.data(), body_of_row.data(), &nbodies,
                                       body_density.data(), n);
        if (rc) return log_printf("rigid bodies: %s\n", dmph_bodies_last_message()), 1;
    }
    if (!ctx) {
        rc = dmph_create(&p, n, type.data(), x.data(), v.data(), &ctx);
        if (rc) return fail("dmph_create", rc, nullptr);
    }
    if (nbodies > 0) {
        rc = dmph_set_bodies(ctx, nbodies, body_of_row.data(), body_density.data());
        if (rc) return fail("dmph_set_bodies", rc, ctx);
        log_printf("rigid bodies: %d\n", nbodies);
    }
    dmph_info info;
    dmph_get_info(ctx, &info);
    log_printf("N0a = %e\nN0p = %e\n", info.n0a, info.n0p);
    log_printf("CellCount[DIM]: %d %d %d\nTotalCellCount: %d\n", info.cell_count[0], info.cell_count[1],
               info.cell_count[2], info.total_cell_count);
    log_printf("CellWidth[DIM]: %e %e %e\n", info.cell_width[0], info.cell_width[1], info.cell_width[2]);
    log_printf("Using GPU %d (%s)\n", gpu, dmph_version());

    // VTK output: the fields of writeVtkFile from the current state
    std::vector<double> kn(n), cn(n), kt(n), ct(n), alpha(n), drag(n), vsp(n), vir(n, 0.0);
    std::vector<int> ncount(n);
    auto write_vtk = [&](const char *fn, bool with_virial) -> int {
        int r = dmph_get_state(ctx, type.data(), x.data(), v.data(), nullptr);
        const struct {
            int id;
            void *out;
        } fields[] = {{DMPH_FIELD_NORMAL_SPRING, kn.data()},       {DMPH_FIELD_NORMAL_DAMPING, cn.data()},
                      {DMPH_FIELD_TANGENTIAL_SPRING, kt.data()},   {DMPH_FIELD_TANGENTIAL_DAMPING, ct.data()},
                      {DMPH_FIELD_NEIGHBOR_COUNT, ncount.data()}, {DMPH_FIELD_ALPHA, alpha.data()},
                      {DMPH_FIELD_DRAG_C, drag.data()},           {DMPH_FIELD_VOL_STRAIN_P, vsp.data()}};
        for (const auto &f : fields)
            if (!r) r = dmph_get_field(ctx, f.id, f.out);
        if (!r && with_virial) r = dmph_get_field(ctx, DMPH_FIELD_VIRIAL_PRESSURE, vir.data());
        if (r) return fail("reading the VTK fields", r, ctx);
        r = dmph_write_vtk_file(fn, n, type.data(), x.data(), v.data(), kn.data(), cn.data(), kt.data(), ct.data(),
                                ncount.data(), alpha.data(), drag.data(), vsp.data(), vir.data());
        if (r) return log_printf("cannot write %s\n", fn), 1;
        return 0;
    };
    // the reference writes this file after initialisation (:426); its virial
    // pressure has not been computed yet and is zero
    if (resumef.empty() && write_vtk("output.vtk", false)) return 1;

    double Time = sched.time, OutputNext = sched.output_next, VtkOutputNext = sched.vtk_output_next;
    const double Dt = p.dt;
    int iStep = resumef.empty() ? (int)(Time / Dt) : sched.step;
    {
        time_t t = time(NULL);
        log_printf("start main roop at %s\n", ctime(&t));
    }
    const clock_t c0 = clock();
    while (Time < p.end_time + 1.0e-5 * Dt) {
        if (Time + 1.0e-5 * Dt >= OutputNext) {
            char fn[1024];
            std::snprintf(fn, sizeof(fn), proff.c_str(), iStep);
            dmph_params hp = p;
            hp.time = Time;
            rc = dmph_get_state(ctx, type.data(), x.data(), v.data(), nullptr);
            if (rc) return fail("dmph_get_state", rc, ctx);
            rc = dmph_write_prof_file(fn, &hp, n, type.data(), x.data(), v.data());
            if (rc) return log_printf("cannot write %s\n", fn), 1;
            log_printf("@ Prof Output Time : %e\n", Time);
            OutputNext += p.output_interval;
            if (checkpoint) {
                const Schedule now = {Time, OutputNext, VtkOutputNext, iStep};
                const std::string ck = std::string(fn) + ".ckpt";
                rc = dmph_checkpoint_write(ctx, ck.c_str(), &now, (int)sizeof(now));
                if (rc) return fail("dmph_checkpoint_write", rc, ctx);
            }
        }
        rc = dmph_step(ctx, 1);
        if (rc) return fail("dmph_step", rc, ctx);
        if (Time + 1.0e-5 * Dt >= VtkOutputNext) {
            char fn[1024];
            std::snprintf(fn, sizeof(fn), vtkf.c_str(), iStep);
            if (write_vtk(fn, true)) return 1;
            log_printf("@ Vtk Output Time : %e\n", Time);
            VtkOutputNext += p.vtk_output_interval;
        }
        Time += Dt;
        iStep++;
    }
    const clock_t c1 = clock();
    dmph_get_info(ctx, &info);
    {
        time_t t = time(NULL);
        log_printf("end main roop at %s\n", ctime(&t));
    }
    log_printf("steps %lld, rebuilds %lld\n", (long long)info.steps, (long long)info.rebuilds);
    log_printf("total:                   %lf [CPU sec]\n", (double)(c1 - c0) / CLOCKS_PER_SEC);
    dmph_destroy(ctx);
    if (g_log) std::fclose(g_log);
    return 0;
}
