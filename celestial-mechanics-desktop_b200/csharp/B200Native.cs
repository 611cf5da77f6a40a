// B200Native.cs - P/Invoke declarations of libnbody_b200 (include/nbody_b200.h).
//
// Added to the desktop app beside its CPU backends
// (src/CelestialMechanics.Physics/Solvers/).  One DllImport per nb_* entry
// point, with the same name, argument order and types: int32_t -> int,
// int64_t -> long, uint64_t -> ulong, uint8_t* -> byte* (a .NET bool[] is one
// byte per element and is passed as byte*, avoiding BOOL marshalling),
// handles and void* -> IntPtr, const char* results -> IntPtr (read with
// Marshal.PtrToStringAnsi).  Every call returns an int status; Check()
// turns a negative one into an exception.  There is no CPU fallback.
using System;
using System.Runtime.InteropServices;

namespace CelestialMechanics.Physics.Solvers;

internal static unsafe class B200Native
{
    private const string Lib = "nbody_b200";

    // enum nb_status
    public const int Ok = 0, ErrInvalidArg = -1, ErrCapacity = -2, ErrCuda = -3, ErrTimeout = -4,
        ErrStackOverflow = -5, ErrNoDevice = -6, ErrNonfinite = -7, ErrState = -8;

    // enum nb_mode and the NB_FLAG_* bits of `flags`
    public const int ModeDirect = 0, ModeDirectFp64 = 1, ModeBarnesHut = 2, ModeBarnesHutRef = 3;
    public const int ModeMask = 0xF;
    public const int FlagShellTheorem = 0x10, FlagNoQuadrupole = 0x20, FlagCollisions = 0x40,
        FlagLearnedMac = 0x80, FlagYoshida4 = 0x100, FlagAdaptiveDt = 0x200,
        FlagOrderSimd = 0x400, FlagOrderPairwise = 0x800;

    // enum nb_param
    public const int ParamTheta = 1, ParamLeafCapacity = 2, ParamMaxMergesFrame = 3,
        ParamMaxMergesBody = 4, ParamMinRadius = 5, ParamDensityMerge = 6, ParamTiming = 7,
        ParamMacBudget = 8, ParamGroupBodies = 9, ParamGroupPack = 10, ParamMacThetaLo = 11,
        ParamMacThetaHi = 12, ParamMacScreenQuantile = 13, ParamEnsDirectShape = 14,
        ParamMacAuditInterval = 15, ParamMacAuditSamples = 16, ParamMacAuditRms = 17,
        ParamAdaptiveEta = 18, ParamAdaptiveDtMin = 19, ParamAdaptiveDtMax = 20,
        ParamGroupSpan = 21, ParamEnsWalkShape = 22;

    // enum nb_timing, enum nb_counter
    public const int TBuild = 0, TTraversal = 1, TTotal = 2, TSort = 3, TTree = 4, TCollide = 5,
        TCount = 6;
    public const int CCellInteractions = 0, CBodyInteractions = 1, CNodes = 2, CActive = 3,
        CPairs = 4, CMerges = 5, COverflows = 6, CGroups = 7, CMaxGroupWork = 8, CMacEvals = 9,
        CMacAudits = 10, CMacFallback = 11, CCount = 12;

    public const int MacParams = 4801, MacNorm = 18, MacScreen = 10, EnsTreeChoices = 11;
    public const int NoAllocSortMax = 1048576;

    // ---- lifetime ---------------------------------------------------------
    [DllImport(Lib)] public static extern int nb_create(int capacity, int device, out IntPtr handle);
    [DllImport(Lib)] public static extern int nb_destroy(IntPtr h);
    [DllImport(Lib)] public static extern IntPtr nb_last_error(IntPtr h);
    [DllImport(Lib)] public static extern int nb_set_param_f64(IntPtr h, int param, double value);
    [DllImport(Lib)] public static extern int nb_set_param_i32(IntPtr h, int param, int value);
    [DllImport(Lib)] public static extern int nb_get_timings(IntPtr h, double* outMs, int n);
    [DllImport(Lib)] public static extern int nb_get_counters(IntPtr h, long* outCounts, int n);
    [DllImport(Lib)] public static extern int nb_get_adaptive_dt(IntPtr h, double* dt);
    [DllImport(Lib)] public static extern int nb_max_acceleration(IntPtr h, double* aMax);
    [DllImport(Lib)] public static extern int nb_get_body_count(IntPtr h, int* n, int* nActive);
    [DllImport(Lib)] public static extern IntPtr nb_stream(IntPtr h);
    [DllImport(Lib)] public static extern IntPtr nb_version();

    // ---- the seam: IPhysicsComputeBackend.ComputeForces ----------------------
    [DllImport(Lib)] public static extern int nb_compute_forces(IntPtr h, int n,
        double* px, double* py, double* pz, double* mass, double* radius, byte* active,
        double softening, int flags, double* ax, double* ay, double* az);

    // ---- device-resident state: ISoAIntegrator -------------------------------
    [DllImport(Lib)] public static extern int nb_set_state(IntPtr h, int n,
        double* px, double* py, double* pz, double* vx, double* vy, double* vz,
        double* mass, double* radius, double* density, byte* active, byte* collidable,
        double* oldAx, double* oldAy, double* oldAz);
    [DllImport(Lib)] public static extern int nb_get_state(IntPtr h, int* nOut,
        double* px, double* py, double* pz, double* vx, double* vy, double* vz,
        double* ax, double* ay, double* az, double* mass, double* radius, byte* active, int* ids);
    [DllImport(Lib)] public static extern int nb_step(IntPtr h, int nSteps, double dt,
        double softening, int flags);
    [DllImport(Lib)] public static extern int nb_diagnostics(IntPtr h, double softening,
        int peMode, double* out13);
    [DllImport(Lib)] public static extern int nb_force_error(IntPtr h, int nSamples, ulong seed,
        double softening, int flags, double* out3);

    // ---- single stages ----------------------------------------------------------
    [DllImport(Lib)] public static extern int nb_morton_keys(IntPtr h, int n, double* px,
        double* py, double* pz, byte* active, int mode, double* cube4, ulong* keys, int* idx,
        double* cube4Out);
    [DllImport(Lib)] public static extern int nb_sort_pairs(IntPtr h, int n, ulong* keys,
        int* values);
    [DllImport(Lib)] public static extern int nb_sort_pairs_noalloc(ulong* keys, int* values,
        int n, IntPtr stream);
    [DllImport(Lib)] public static extern int nb_build_octree(IntPtr h, int n, double* px,
        double* py, double* pz, double* mass, byte* active, double* cube4, int leafCapacity,
        int maxNodes, int* nNodes, int* level, int* firstChild, int* nChildren, int* bodyFirst,
        int* bodyCount, double* nodeMass, double* com3, float* quad6, int* sortedIdx,
        ulong* sortedKeys);
    [DllImport(Lib)] public static extern int nb_compact_indices(IntPtr h, int n, byte* active,
        double* mass, int* dest, int* nKept);
    [DllImport(Lib)] public static extern int nb_broad_phase(IntPtr h, int n, double* px,
        double* py, double* pz, double* radius, byte* active, byte* collidable, int maxPairs,
        int* pairLo, int* pairHi, int* nPairs);

    // ---- learned multipole acceptance criterion ---------------------------------
    [DllImport(Lib)] public static extern int nb_mac_harvest(IntPtr h, int maxRecords,
        double sampleFrac, ulong seed, double softening, int* nAdded);
    [DllImport(Lib)] public static extern int nb_mac_dataset(IntPtr h, int* n, float* x, float* y);
    [DllImport(Lib)] public static extern int nb_mac_clear(IntPtr h);
    [DllImport(Lib)] public static extern int nb_mac_train(IntPtr h, int epochs, int batch,
        double lr, ulong seed, double* lossPerEpoch);
    [DllImport(Lib)] public static extern int nb_mac_set_params(IntPtr h, float* p, int n);
    [DllImport(Lib)] public static extern int nb_mac_get_params(IntPtr h, float* p, int n);
    [DllImport(Lib)] public static extern int nb_mac_gradient(IntPtr h, float* x, float* y, int n,
        float* grad, double* loss);
    [DllImport(Lib)] public static extern int nb_mac_predict(IntPtr h, float* x, int n, float* y);
    [DllImport(Lib)] public static extern int nb_mac_audit_state(IntPtr h, double* rms,
        double* maxErr, long* audits, int* fallback);
    [DllImport(Lib)] public static extern int nb_mac_fit_screen(IntPtr h);
    [DllImport(Lib)] public static extern int nb_mac_get_screen(IntPtr h, float* s, int n);
    [DllImport(Lib)] public static extern int nb_mac_set_screen(IntPtr h, float* s, int n);

    // ---- batched ensembles ---------------------------------------------------------
    [DllImport(Lib)] public static extern int nb_ens_create(int nSystems, int* sizes, int dsMaxN,
        int device, out IntPtr handle);
    [DllImport(Lib)] public static extern int nb_ens_destroy(IntPtr h);
    [DllImport(Lib)] public static extern IntPtr nb_ens_last_error(IntPtr h);
    [DllImport(Lib)] public static extern int nb_ens_info(IntPtr h, long* outInfo, int n);
    [DllImport(Lib)] public static extern int nb_ens_set_param_f64(IntPtr h, int param, double value);
    [DllImport(Lib)] public static extern int nb_ens_set_param_i32(IntPtr h, int param, int value);
    [DllImport(Lib)] public static extern int nb_ens_set_state(IntPtr h, double* px, double* py,
        double* pz, double* vx, double* vy, double* vz, double* mass);
    [DllImport(Lib)] public static extern int nb_ens_get_state(IntPtr h, double* px, double* py,
        double* pz, double* vx, double* vy, double* vz, double* ax, double* ay, double* az);
    [DllImport(Lib)] public static extern int nb_ens_compute_forces(IntPtr h, double softening);
    [DllImport(Lib)] public static extern int nb_ens_step(IntPtr h, int nSteps, double dt,
        double softening);
    [DllImport(Lib)] public static extern int nb_ens_autotune(IntPtr h, double softening,
        int* shape, double* msPerShape);
    [DllImport(Lib)] public static extern int nb_ens_autotune_tree(IntPtr h, double softening,
        int* choice, double* msPerChoice);
    [DllImport(Lib)] public static extern int nb_ens_force_error(IntPtr h, int samples, ulong seed,
        double softening, double* rms, double* maxErr);
    [DllImport(Lib)] public static extern int nb_ens_energy(IntPtr h, double softening,
        double* energy, double* kinetic, double* potential);
    [DllImport(Lib)] public static extern int nb_ens_get_counters(IntPtr h, long* outCounts, int n);
    [DllImport(Lib)] public static extern int nb_ens_get_timings(IntPtr h, double* msPerStep);

    /// <summary>Throws when <paramref name="status"/> is an error, with the
    /// handle's last error message (the convention of the reference's native
    /// API, native_api.cpp:30-55, mapped onto exceptions as
    /// CudaPhysicsBackend does).</summary>
    public static void Check(IntPtr h, int status)
    {
        if (status == Ok) return;
        string msg = h != IntPtr.Zero ? Marshal.PtrToStringAnsi(nb_last_error(h)) ?? "" : "";
        throw new InvalidOperationException($"nbody_b200 status {status}: {msg}");
    }
}
