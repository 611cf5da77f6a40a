// B200BackendSelection.cs - the one branch NBodySolver.SelectBackend needs.
//
// NBodySolver.SelectBackend (src/CelestialMechanics.Physics/Solvers/
// NBodySolver.cs:451-484) picks the force backend from PhysicsConfig.  The
// maintainer adds the settings below to the solver's configuration
// (PhysicsConfig.cs:41-85 holds the others) and, as the first branch of
// SelectBackend:
//
//     if (_b200.Enabled)
//         backend = _b200.Resolve(_soaBodies.Capacity, _useBarnesHut, _theta,
//                                 _useSimd, _deterministicMode, _useParallel);
//
// The existing `backend is IGravityModelAwareBackend` line then sets the
// shell theorem on it as on every CPU backend.
using System;

namespace CelestialMechanics.Physics.Solvers;

public sealed class B200BackendSelection : IDisposable
{
    private B200PhysicsBackend? _backend;

    /// <summary>Use the B200 engine for forces.</summary>
    public bool Enabled { get; set; }
    /// <summary>CUDA device ordinal.</summary>
    public int Device { get; set; }
    /// <summary>All-pairs forces in FP64 (bit-identical to the CPU backend the
    /// app would have picked) instead of FP32 pair forces.</summary>
    public bool Fp64DirectSum { get; set; }
    /// <summary>Learned opening criterion in Barnes-Hut mode.</summary>
    public bool UseLearnedMac { get; set; }
    public double MacBudget { get; set; } = -3.0;

    /// <summary>The backend for the solver's current settings; the handle is
    /// created once, at the first call, and recreated when the capacity grows.</summary>
    public B200PhysicsBackend Resolve(int capacity, bool useBarnesHut, double theta, bool useSimd,
        bool deterministic, bool useParallel)
    {
        if (_backend == null || _backend.Capacity < capacity)
        {
            _backend?.Dispose();
            _backend = new B200PhysicsBackend(capacity, Device);
        }
        _backend.Theta = theta;
        _backend.UseLearnedMac = UseLearnedMac;
        _backend.MacBudget = MacBudget;
        if (useBarnesHut)
        {
            _backend.Mode = B200ForceMode.BarnesHut;
        }
        else if (Fp64DirectSum)
        {
            _backend.Mode = B200ForceMode.DirectFp64;
            // the bits of the CPU backend SelectBackend would choose: SIMD,
            // else single-thread when deterministic or not parallel, else
            // CpuParallel (NBodySolver.cs:461-471)
            _backend.SummationOrder = useSimd ? B200SummationOrder.Simd
                : (deterministic || !useParallel) ? B200SummationOrder.SingleThread
                : B200SummationOrder.CpuParallel;
        }
        else
        {
            _backend.Mode = B200ForceMode.Direct;
        }
        return _backend;
    }

    public void Dispose() => _backend?.Dispose();
}
