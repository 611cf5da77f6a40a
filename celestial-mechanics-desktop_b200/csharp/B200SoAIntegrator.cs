// B200SoAIntegrator.cs - velocity Verlet on the GPU behind ISoAIntegrator.
//
// ISoAIntegrator.Step (src/CelestialMechanics.Physics/Integrators/
// ISoAIntegrator.cs) with SoAVerletIntegrator's arithmetic
// (SoAVerletIntegrator.cs:48-116): half kick with OldAcc, drift, forces, half
// kick, OldAcc = Acc.  With a B200PhysicsBackend the whole step runs on the
// device (nb_set_state, nb_step, nb_get_state); the FP64 direct-sum modes
// give the CPU integrator's trajectory bit for bit.  NBodySolver refreshes
// the SoA from its bodies before every step (NBodySolver.cs:383-391), so
// Step uploads the state each call; StepMany keeps it on the device for a
// batch of steps (benchmarks, headless runs) and downloads once.  With any
// other backend Step runs SoAVerletIntegrator itself, unchanged.
using System;
using CelestialMechanics.Physics.SoA;
using CelestialMechanics.Physics.Solvers;

namespace CelestialMechanics.Physics.Integrators;

public sealed unsafe class B200SoAIntegrator : ISoAIntegrator
{
    private readonly SoAVerletIntegrator _cpu = new();

    /// <inheritdoc/>
    public string Name => "Verlet-SoA (B200)";

    /// <summary>Yoshida's 4th-order composition instead of one Verlet step
    /// (three force evaluations per step).</summary>
    public bool Yoshida4 { get; set; }

    /// <inheritdoc/>
    public void Step(BodySoA bodies, IPhysicsComputeBackend backend, double softening, double dt)
    {
        if (backend is B200PhysicsBackend gpu) StepMany(bodies, gpu, softening, dt, 1);
        else _cpu.Step(bodies, backend, softening, dt);
    }

    /// <summary><paramref name="steps"/> steps with the state resident on the
    /// device; the bodies are uploaded once and downloaded once.</summary>
    public void StepMany(BodySoA bodies, B200PhysicsBackend gpu, double softening, double dt,
        int steps)
    {
        IntPtr h = gpu.Handle;
        int n = bodies.Count;
        gpu.ApplyParams();
        int flags = gpu.Flags() | (Yoshida4 ? B200Native.FlagYoshida4 : 0);
        fixed (double* px = bodies.PosX, py = bodies.PosY, pz = bodies.PosZ,
                      vx = bodies.VelX, vy = bodies.VelY, vz = bodies.VelZ,
                      ax = bodies.AccX, ay = bodies.AccY, az = bodies.AccZ,
                      oax = bodies.OldAccX, oay = bodies.OldAccY, oaz = bodies.OldAccZ,
                      m = bodies.Mass, r = bodies.Radius, rho = bodies.Density)
        fixed (bool* act = bodies.IsActive, col = bodies.IsCollidable)
        {
            B200Native.Check(h, B200Native.nb_set_state(h, n, px, py, pz, vx, vy, vz, m, r, rho,
                (byte*)act, (byte*)col, oax, oay, oaz));
            B200Native.Check(h, B200Native.nb_step(h, steps, dt, softening, flags));
            int nOut = 0;
            B200Native.Check(h, B200Native.nb_get_state(h, &nOut, px, py, pz, vx, vy, vz,
                ax, ay, az, null, null, null, null));
        }
        // OldAcc = Acc, ready for the next call (SoAVerletIntegrator's rotate)
        Array.Copy(bodies.AccX, bodies.OldAccX, n);
        Array.Copy(bodies.AccY, bodies.OldAccY, n);
        Array.Copy(bodies.AccZ, bodies.OldAccZ, n);
        gpu.ReadTimings();
    }
}
