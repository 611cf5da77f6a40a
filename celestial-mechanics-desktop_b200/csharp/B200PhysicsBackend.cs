// B200PhysicsBackend.cs - the B200 engine behind the app's force-backend seam.
//
// Sits beside CpuParallelBackend (src/CelestialMechanics.Physics/Solvers/).
// Same contract as IPhysicsComputeBackend.ComputeForces
// (IPhysicsComputeBackend.cs:21-34): AccX/Y/Z are written for every row in
// [0, Count); active rows get the softened sum over the other active bodies,
// inactive rows get 0.  Implements IGravityModelAwareBackend so that
// NBodySolver.SelectBackend sets EnableShellTheorem on it as on the CPU
// backends (NBodySolver.cs:476-477), and exposes the timing properties the
// benchmark reads from BarnesHutBackend (BarnesHutBackend.cs:101-107,
// PhysicsBenchmark.cs:225-249).  One handle = one CUDA stream and its device
// buffers; like the CPU backends the object is used from one thread.
using System;
using CelestialMechanics.Physics.SoA;

namespace CelestialMechanics.Physics.Solvers;

/// <summary>Which CPU backend's bits the FP64 direct sum reproduces.</summary>
public enum B200SummationOrder
{
    /// <summary>CpuParallelBackend (coefficient ((m*inv)*inv)*inv).</summary>
    CpuParallel = 0,
    /// <summary>SimdSingleThreadBackend and the native engine's CPU brute force.</summary>
    Simd = B200Native.FlagOrderSimd,
    /// <summary>CpuSingleThreadBackend's Newton's-third-law loop.</summary>
    SingleThread = B200Native.FlagOrderPairwise,
}

/// <summary>How the forces are evaluated on the GPU.</summary>
public enum B200ForceMode
{
    /// <summary>Barnes-Hut group walk, monopole + quadrupole, FP32 pair forces
    /// on FP64-differenced coordinates (rms force error ~2e-4 at theta 0.5).</summary>
    BarnesHut = B200Native.ModeBarnesHut,
    /// <summary>The reference solver's semantics (monopole, its MAC), FP64.</summary>
    BarnesHutReference = B200Native.ModeBarnesHutRef,
    /// <summary>All pairs, FP32 pair forces on FP64-differenced coordinates.</summary>
    Direct = B200Native.ModeDirect,
    /// <summary>All pairs in FP64, bit-identical to the CPU backend that
    /// <see cref="B200PhysicsBackend.SummationOrder"/> names.</summary>
    DirectFp64 = B200Native.ModeDirectFp64,
}

public sealed unsafe class B200PhysicsBackend : IPhysicsComputeBackend, IGravityModelAwareBackend,
    IDisposable
{
    private IntPtr _h;
    private readonly int _capacity;
    private readonly double[] _timings = new double[B200Native.TCount];

    public bool EnableShellTheorem { get; set; }
    public B200ForceMode Mode { get; set; } = B200ForceMode.BarnesHut;
    public B200SummationOrder SummationOrder { get; set; } = B200SummationOrder.CpuParallel;
    /// <summary>Barnes-Hut opening angle (PhysicsConfig.Theta).</summary>
    public double Theta { get; set; } = 0.5;
    /// <summary>Learned opening criterion (needs a network: see
    /// <see cref="LoadNetwork"/>); only in <see cref="B200ForceMode.BarnesHut"/>
    /// without the shell theorem.</summary>
    public bool UseLearnedMac { get; set; }
    /// <summary>log10 of the tolerated relative force error per cell (learned MAC).</summary>
    public double MacBudget { get; set; } = -3.0;

    public double LastBuildTimeMs { get; private set; }
    public double LastTraversalTimeMs { get; private set; }
    public double LastTotalTimeMs { get; private set; }

    /// <summary>Native handle, for <see cref="B200SoAIntegrator"/>.</summary>
    internal IntPtr Handle => _h;
    public int Capacity => _capacity;

    public B200PhysicsBackend(int capacity, int device = 0)
    {
        _capacity = capacity;
        B200Native.Check(IntPtr.Zero, B200Native.nb_create(capacity, device, out _h));
    }

    /// <summary>The nb_* flags for the current settings (also used by the
    /// device-resident integrator).</summary>
    internal int Flags()
    {
        int flags = (int)Mode;
        if (EnableShellTheorem) flags |= B200Native.FlagShellTheorem;
        if (Mode == B200ForceMode.DirectFp64) flags |= (int)SummationOrder;
        if (UseLearnedMac && Mode == B200ForceMode.BarnesHut && !EnableShellTheorem)
            flags |= B200Native.FlagLearnedMac;
        return flags;
    }

    internal void ApplyParams()
    {
        B200Native.Check(_h, B200Native.nb_set_param_f64(_h, B200Native.ParamTheta, Theta));
        B200Native.Check(_h, B200Native.nb_set_param_f64(_h, B200Native.ParamMacBudget, MacBudget));
    }

    public void ComputeForces(BodySoA bodies, double softening)
    {
        if (_h == IntPtr.Zero) throw new ObjectDisposedException(nameof(B200PhysicsBackend));
        if (bodies.Count > _capacity)
            throw new ArgumentException($"{bodies.Count} bodies exceed the backend capacity {_capacity}");
        ApplyParams();
        int flags = Flags();
        fixed (double* px = bodies.PosX, py = bodies.PosY, pz = bodies.PosZ, m = bodies.Mass,
                      r = bodies.Radius, ax = bodies.AccX, ay = bodies.AccY, az = bodies.AccZ)
        fixed (bool* act = bodies.IsActive)
        {
            B200Native.Check(_h, B200Native.nb_compute_forces(_h, bodies.Count, px, py, pz, m, r,
                (byte*)act, softening, flags, ax, ay, az));
        }
        ReadTimings();
    }

    internal void ReadTimings()
    {
        fixed (double* t = _timings)
            B200Native.Check(_h, B200Native.nb_get_timings(_h, t, B200Native.TCount));
        LastBuildTimeMs = _timings[B200Native.TBuild];
        LastTraversalTimeMs = _timings[B200Native.TTraversal];
        LastTotalTimeMs = _timings[B200Native.TTotal];
    }

    /// <summary>Loads a trained learned-MAC network (parameters and screen
    /// saved from <see cref="SaveNetwork"/>).</summary>
    public void LoadNetwork(float[] parameters, float[] screen)
    {
        fixed (float* p = parameters)
            B200Native.Check(_h, B200Native.nb_mac_set_params(_h, p, parameters.Length));
        fixed (float* s = screen)
            B200Native.Check(_h, B200Native.nb_mac_set_screen(_h, s, screen.Length));
    }

    public (float[] Parameters, float[] Screen) SaveNetwork()
    {
        var p = new float[B200Native.MacParams + B200Native.MacNorm];
        var s = new float[B200Native.MacScreen];
        fixed (float* pp = p)
            B200Native.Check(_h, B200Native.nb_mac_get_params(_h, pp, p.Length));
        fixed (float* ps = s)
            B200Native.Check(_h, B200Native.nb_mac_get_screen(_h, ps, s.Length));
        return (p, s);
    }

    public void Dispose()
    {
        if (_h != IntPtr.Zero)
        {
            B200Native.nb_destroy(_h);
            _h = IntPtr.Zero;
        }
    }
}
