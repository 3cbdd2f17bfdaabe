// Reference harness: appended (by oracle/Makefile) to the reference solver's own
// translation unit, source/DEM-MPH.cpp, whose `main` is renamed to
// `dmph_reference_main`.  It is test infrastructure only: it drives the
// reference's file-static functions in the order of the reference main loop
// (source/DEM-MPH.cpp:419-426 for initialisation, :438-581 for one step) and
// dumps every per-particle array at full FP64 precision so that the oracle
// restatement in oracle/dmph_oracle.c can be pinned against the real thing.
//
// Usage:
//   ref_dump <dem.data> <file.grid> <out_dir> <nsteps> [dump_steps...]
//       dumps state after initialisation (step 0) and after each listed step
//   ref_dump --bench <dem.data> <file.grid> <steps> <warmup>
//       times <steps> reference steps (after <warmup> untimed ones) with
//       omp_get_wtime and prints one JSON line, with the time spent in the
//       neighbour rebuilds (calculateCellParticle + calculateNeighbor) of the
//       timed steps and of the initialisation reported apart
#include <string>
#include <vector>
#include <sys/stat.h>
#include <sys/types.h>

static int HarnessDemSteps = 0;
static int HarnessRebuilds = 0;
static double HarnessRebuildSeconds = 0.0;  // wall time of the rebuilds inside harness_step
static double HarnessInitRebuildSeconds = 0.0;  // wall time of the initial cell sort + neighbour build

static void harness_init(const char *data, const char *grid)
{
    log_open("/dev/null");
    readDataFile((char *)data);
    readGridFile((char *)grid);
    initializeWeight();
    initializeFluid();
    initializeWall();
    initializeDomain();
    const double r0 = omp_get_wtime();
    calculateCellParticle();
    calculateNeighbor();
    HarnessInitRebuildSeconds = omp_get_wtime() - r0;
    calculateDensityA();
    calculateGravityCenter();
    calculateDensityP();
    HarnessDemSteps = Dt / DEMDt;  // same conversion as source/DEM-MPH.cpp:434
}

// One iteration of the reference main loop body without file output
// (source/DEM-MPH.cpp:450-579).
static void harness_step()
{
    calculateConvection();
    calculateWall();
    calculatePeriodicBoundary();
    resetForce();
    if (neighborCalculation() == 1) {
        const double r0 = omp_get_wtime();
        freeNeighbor();
        calculateCellParticle();
        calculateNeighbor();
        HarnessRebuildSeconds += omp_get_wtime() - r0;
        HarnessRebuilds++;
    }
    calculateDensityA();
    calculateGravityCenter();
    calculateDensityP();
    calculateDivergenceP();
    calculatePhysicalCoefficients();
    calculateDragForce();
    calculatePressureP();
    calculatePressureA();
    calculateDiffuseInterface();
    calculateViscosityV();
    calculateDragForce();
    calculateBuoyancyForce();
    calculateGravity();
    calculateAcceleration();
    for (int i = 0; i < HarnessDemSteps; i++) {
        calculateNormalDirectionCoefficient();
        calculateTangentialDirectionCoefficient();
        calculateInertialTensor();
        calculateTorque();
        calculateNormalDirectionForce();
        calculateTangentialDirectionForce();
        calculateDEMconvection();
    }
    Time += Dt;
}

static void dump_raw(const std::string &dir, const char *name, const void *p, size_t bytes)
{
    std::string path = dir + "/" + name;
    FILE *f = ::fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    if (bytes) fwrite(p, 1, bytes, f);
    fclose(f);
}

static void harness_dump(const std::string &dir)
{
    mkdir(dir.c_str(), 0755);
    const size_t N = (size_t)ParticleCount;
    const size_t T = (size_t)TotalCellCount;
    dump_raw(dir, "ParticleIndex.i32", ParticleIndex, N * 4);
    dump_raw(dir, "Property.i32", Property, N * 4);
    dump_raw(dir, "Position.f64", Position, N * 24);
    dump_raw(dir, "Velocity.f64", Velocity, N * 24);
    dump_raw(dir, "Force.f64", Force, N * 24);
    dump_raw(dir, "Mass.f64", Mass, N * 8);
    dump_raw(dir, "Kappa.f64", Kappa, N * 8);
    dump_raw(dir, "VolStrainP.f64", VolStrainP, N * 8);
    dump_raw(dir, "DivergenceP.f64", DivergenceP, N * 8);
    dump_raw(dir, "PressureP.f64", PressureP, N * 8);
    dump_raw(dir, "DensityA.f64", DensityA, N * 8);
    dump_raw(dir, "GravityCenter.f64", GravityCenter, N * 24);
    dump_raw(dir, "PressureA.f64", PressureA, N * 8);
    dump_raw(dir, "NormalSpringConstant.f64", NormalSpringConstant, N * 8);
    dump_raw(dir, "NormalViscousDampingConstant.f64", NormalViscousDampingConstant, N * 8);
    dump_raw(dir, "TangentialSpringConstant.f64", TangentialSpringConstant, N * 8);
    dump_raw(dir, "TangentialViscousDampingConstant.f64", TangentialViscousDampingConstant, N * 8);
    dump_raw(dir, "alpha.f64", alpha, N * 8);
    dump_raw(dir, "DragC.f64", DragC, N * 8);
    // the output-cadence virial stress of the state being dumped
    // (calculateVirialStressAtParticle writes only the two virial arrays)
    calculateVirialStressAtParticle();
    dump_raw(dir, "VirialPressure.f64", VirialPressureAtParticle, N * 8);
    dump_raw(dir, "NeighborCount.i32", NeighborCount, N * 4);
    dump_raw(dir, "FluidNeighborCount.i32", FluidNeighborCount, N * 4);
    dump_raw(dir, "SolidNeighborCount.i32", SolidNeighborCount, N * 4);
    dump_raw(dir, "NeighborPtr.i64", NeighborPtr, (N + 1) * 8);
    dump_raw(dir, "NeighborInd.i32", NeighborInd, (size_t)NeighborIndCount * 4);
    dump_raw(dir, "NeighborCalculatedPosition.f64", NeighborCalculatedPosition, N * 24);
    dump_raw(dir, "CellIndex.i32", CellIndex, (size_t)PowerParticleCount * 4);
    dump_raw(dir, "CellParticle.i32", CellParticle, (size_t)PowerParticleCount * 4);
    dump_raw(dir, "CellFluidParticleBegin.i32", CellFluidParticleBegin, T * 4);
    dump_raw(dir, "CellFluidParticleEnd.i32", CellFluidParticleEnd, T * 4);
    dump_raw(dir, "CellSolidParticleBegin.i32", CellSolidParticleBegin, T * 4);
    dump_raw(dir, "CellSolidParticleEnd.i32", CellSolidParticleEnd, T * 4);
    dump_raw(dir, "CellWallParticleBegin.i32", CellWallParticleBegin, T * 4);
    dump_raw(dir, "CellWallParticleEnd.i32", CellWallParticleEnd, T * 4);

    std::string meta = dir + "/meta.txt";
    FILE *f = ::fopen(meta.c_str(), "w");
    fprintf(f, "Time %.17g\n", Time);
    fprintf(f, "ParticleCount %d\n", ParticleCount);
    fprintf(f, "PowerParticleCount %d\n", PowerParticleCount);
    fprintf(f, "TotalCellCount %d\n", TotalCellCount);
    fprintf(f, "CellCount %d %d %d\n", CellCount[0], CellCount[1], CellCount[2]);
    fprintf(f, "CellWidth %.17g %.17g %.17g\n", CellWidth[0], CellWidth[1], CellWidth[2]);
    fprintf(f, "N0a %.17g\nN0p %.17g\nR2g %.17g\n", N0a, N0p, R2g);
    fprintf(f, "Swa %.17g\nSwg %.17g\nSwp %.17g\nSwv %.17g\n", Swa, Swg, Swp, Swv);
    fprintf(f, "MaxRadius %.17g\n", MaxRadius);
    fprintf(f, "FluidRange %d %d\n", FluidParticleBegin, FluidParticleEnd);
    fprintf(f, "SolidRange %d %d\n", SolidParticleBegin, SolidParticleEnd);
    fprintf(f, "WallRange %d %d\n", WallParticleBegin, WallParticleEnd);
    fprintf(f, "NeighborIndCount %ld\n", NeighborIndCount);
    fprintf(f, "DemSteps %d\n", HarnessDemSteps);
    fprintf(f, "Rebuilds %d\n", HarnessRebuilds);
    fprintf(f, "CofK %.17g\n", CofK);
    for (int t = 0; t < TYPE_COUNT; t++) fprintf(f, "CofA%d %.17g\n", t, CofA[t]);
    fclose(f);
}

int main(int argc, char **argv)
{
    if (argc >= 6 && std::string(argv[1]) == "--bench") {
        harness_init(argv[2], argv[3]);
        const int steps = atoi(argv[4]);
        const int warmup = atoi(argv[5]);
        for (int i = 0; i < warmup; i++) harness_step();
        const int rebuilds0 = HarnessRebuilds;
        const double rs0 = HarnessRebuildSeconds;
        const double t0 = omp_get_wtime();
        for (int i = 0; i < steps; i++) harness_step();
        const double t1 = omp_get_wtime();
        printf("{\"particles\": %d, \"steps\": %d, \"seconds\": %.6f, \"threads\": %d, "
               "\"rebuilds\": %d, \"rebuild_seconds\": %.6f, \"init_rebuild_seconds\": %.6f, "
               "\"dem_substeps\": %d}\n",
               ParticleCount, steps, t1 - t0, omp_get_max_threads(), HarnessRebuilds - rebuilds0,
               HarnessRebuildSeconds - rs0, HarnessInitRebuildSeconds, HarnessDemSteps);
        return 0;
    }
    if (argc < 5) {
        fprintf(stderr, "usage: %s data grid out_dir nsteps [dump_steps...]\n", argv[0]);
        return 1;
    }
    harness_init(argv[1], argv[2]);
    const std::string out = argv[3];
    mkdir(out.c_str(), 0755);
    const int nsteps = atoi(argv[4]);
    std::vector<int> dumps;
    for (int a = 5; a < argc; a++) dumps.push_back(atoi(argv[a]));
    harness_dump(out + "/step0");
    for (int s = 1; s <= nsteps; s++) {
        harness_step();
        for (int d : dumps)
            if (d == s) harness_dump(out + "/step" + std::to_string(s));
    }
    return 0;
}
