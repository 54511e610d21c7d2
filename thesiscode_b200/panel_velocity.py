"""Host mirror of PanelVelocityParallelModule (PanelVelocityParallel.f90:1-20).

Same public names, argument meaning and state as the Fortran module:

    BVERK4(aParticles, aPanels, dt, procRank, numProcs)   :435-658
    InitializeMPIRK4 / FinalizeMPIRK4 / LoadBalance        :126-230
    ResetRK4, SetSmooth, GetSmooth, ResetArea              :96-120, :321
    totalKE, kineticEnergy                                 :25-26

The module's `save` state lives in a `PanelVelocity` object (one per rank
and device); the module-level functions act on a default instance exactly
like the Fortran module's globals. Every sum runs in libthesiscode_b200 on
the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .grid import GatherMaps, Panels, Particles, gather_panels, scatter_panels

PRECISIONS = {"fp64": N.TC_FP64, "fp32c": N.TC_FP32C}


def load_balance(n: int, num_procs: int) -> tuple[np.ndarray, np.ndarray]:
    """LoadBalance (PanelVelocityParallel.f90:182-204): contiguous chunks of n // p, the last
    rank takes the remainder. Returns 0-based half-open (start, end) per rank."""
    if num_procs < 1:
        raise ValueError("numProcs must be >= 1")
    chunk = n // num_procs
    start = np.arange(num_procs, dtype=np.int64) * chunk
    end = start + chunk
    end[-1] = n
    return start, end


class Context:
    """Owns one tc_ctx (device, precision, Omega, deltas, device-resident RK4 state)."""

    def __init__(self, device: int = 0, precision: str | int = "fp64"):
        prec = PRECISIONS.get(precision, precision)
        h = ctypes.c_void_p()
        N.call("tc_create", int(device), int(prec), ctypes.byref(h))
        self._h = h
        self.device = device

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._h is None:
            raise RuntimeError("context destroyed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            N.lib().tc_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    # parameters -----------------------------------------------------------
    def set_omega(self, omega: float) -> None:
        N.call("tc_set_omega", self.handle, float(omega))

    def get_omega(self) -> float:
        v = ctypes.c_double()
        N.call("tc_get_omega", self.handle, ctypes.byref(v))
        return v.value

    def set_deltas(self, active: float, vertex: float, passive: float) -> None:
        N.call("tc_set_deltas", self.handle, float(active), float(vertex), float(passive))

    def get_deltas(self) -> tuple[float, float, float]:
        v = (ctypes.c_double * 3)()
        N.call("tc_get_deltas", self.handle, v)
        return tuple(v)

    def set_precision(self, precision) -> None:
        N.call("tc_set_precision", self.handle, int(PRECISIONS.get(precision, precision)))

    def set_stream(self, stream_ptr: int) -> None:
        N.call("tc_set_stream", self.handle, ctypes.c_void_p(stream_ptr))

    def synchronize(self) -> None:
        N.call("tc_synchronize", self.handle)

    # one sum (host arrays) ------------------------------------------------
    def velocity(self, target_class: int, X, src_x, vort, area, i0=0, i1=None):
        """One of BVEActiveRHS / BVEPassiveRHS / BVESmoothVelocity on host arrays.
        Returns (dX (m,3), dVort (m,) or None)."""
        src_x = np.ascontiguousarray(src_x, dtype=np.float64)
        vort = np.ascontiguousarray(vort, dtype=np.float64)
        area = np.ascontiguousarray(area, dtype=np.float64)
        n = src_x.shape[0]
        if target_class == N.TC_ACTIVE:
            Xc, m = None, n
        else:
            Xc = np.ascontiguousarray(X, dtype=np.float64)
            m = Xc.shape[0]
        i1 = m if i1 is None else i1
        dX = np.zeros((m, 3))
        dV = np.zeros(m) if target_class == N.TC_ACTIVE else None
        N.call("tc_bs_velocity", self.handle, int(target_class), N.dptr(Xc), m, N.dptr(src_x),
               N.dptr(vort), N.dptr(area), n, int(i0), int(i1), N.dptr(dX), N.dptr(dV))
        return dX, dV

    # RK4 (host arrays, in place) -----------------------------------------------
    def rk4_step(self, xA, zetaA, areaA, xV, xQ, dt: float, nsteps: int = 1):
        """nsteps fused RK4 steps on host arrays (updated in place).
        Returns (totalKE per step, kineticEnergy of the last step)."""
        for a in (xA, zetaA, areaA, xV, xQ):
            if not (a.dtype == np.float64 and a.flags.c_contiguous):
                raise TypeError("RK4 arrays must be C-contiguous float64")
        tke = np.zeros(max(nsteps, 1))
        ke = np.zeros(xA.shape[0])
        N.call("tc_rk4_step", self.handle, N.dptr(xA), N.dptr(zetaA), N.dptr(areaA), xA.shape[0],
               N.dptr(xV), xV.shape[0], N.dptr(xQ), xQ.shape[0], float(dt), int(nsteps),
               N.dptr(tke), N.dptr(ke))
        return tke[:nsteps], ke

    def strat_rk4_step(self, xA, absVortA, areaA, xV, xQ, t: float, dt: float, nsteps: int = 1,
                       absVortV=None):
        """nsteps forced (stratosphere) RK4 steps from time t on host arrays (positions updated in
        place). Returns (relVortA, relVortV or None, totalKE per step, kineticEnergy)."""
        for a in (xA, areaA, xV, xQ):
            if not (a.dtype == np.float64 and a.flags.c_contiguous):
                raise TypeError("RK4 arrays must be C-contiguous float64")
        absA = np.ascontiguousarray(absVortA, dtype=np.float64)
        absV = None if absVortV is None else np.ascontiguousarray(absVortV, dtype=np.float64)
        relA = np.zeros(xA.shape[0])
        relV = None if absV is None else np.zeros(xV.shape[0])
        tke = np.zeros(max(nsteps, 1))
        ke = np.zeros(xA.shape[0])
        N.call("tc_strat_rk4_step", self.handle, N.dptr(xA), N.dptr(absA), N.dptr(relA), N.dptr(areaA),
               xA.shape[0], N.dptr(xV), N.dptr(absV), N.dptr(relV), xV.shape[0], N.dptr(xQ), xQ.shape[0],
               float(t), float(dt), int(nsteps), N.dptr(tke), N.dptr(ke))
        return relA, relV, tke[:nsteps], ke

    def reset_rk4(self) -> None:
        N.call("tc_reset_rk4", self.handle)

    # device-resident state, checkpoints ------------------------------------------
    def rk4_load(self, xA, zetaA, areaA, xV, xQ) -> None:
        """Copy a state (host arrays) to the device (tc_rk4_load)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (xA, zetaA, areaA, xV, xQ)]
        N.call("tc_rk4_load", self.handle, N.dptr(arrs[0]), N.dptr(arrs[1]), N.dptr(arrs[2]),
               arrs[0].shape[0], N.dptr(arrs[3]), arrs[3].shape[0], N.dptr(arrs[4]),
               arrs[4].shape[0], 0)

    def rk4_advance(self, dt: float, nsteps: int) -> np.ndarray:
        """nsteps RK4 steps of the device-resident state; returns totalKE per step."""
        tke = np.zeros(max(nsteps, 1))
        N.call("tc_rk4_advance", self.handle, float(dt), int(nsteps), N.dptr(tke))
        return tke[:nsteps]

    def rk4_store(self, nA: int, nV: int, nQ: int) -> tuple:
        """The device-resident state as host arrays (xA, zetaA, xV, xQ)."""
        xA, zA, xV, xQ = np.zeros((nA, 3)), np.zeros(nA), np.zeros((nV, 3)), np.zeros((nQ, 3))
        N.call("tc_rk4_store", self.handle, N.dptr(xA), N.dptr(zA), N.dptr(xV), N.dptr(xQ), None, 0)
        return xA, zA, xV, xQ

    def save_state(self, path) -> None:
        """Checkpoint the device-resident state to `path` (tc_rk4_save)."""
        N.call("tc_rk4_save", self.handle, str(path).encode())

    def restore_state(self, path) -> None:
        """Load a checkpoint written by save_state (tc_rk4_restore)."""
        N.call("tc_rk4_restore", self.handle, str(path).encode())

    def steps_done(self) -> int:
        """Steps advanced since the state was loaded, counting a restored checkpoint's."""
        v = ctypes.c_longlong()
        N.call("tc_rk4_steps_done", self.handle, ctypes.byref(v))
        return v.value


class PanelVelocity:
    """The `save` state of PanelVelocityParallelModule for one rank."""

    def __init__(self, device: int = 0, precision: str | int = "fp64"):
        self.ctx = Context(device, precision)
        self.totalKE = 0.0
        self.kineticEnergy = None
        self._maps: GatherMaps | None = None
        self._ranges = None
        self._mpi_ready = False
        self.reset_areas = False

    # User decisions (:96-120)
    def SetSmooth(self, new_smooth: float) -> None:
        self.ctx.set_deltas(*self.ctx.get_deltas()[:2], new_smooth)

    def GetSmooth(self) -> float:
        return self.ctx.get_deltas()[2]

    def GetOmega(self) -> float:
        return self.ctx.get_omega()

    def SetOmega(self, omega: float) -> None:
        """SetOmega (TracerAndVorticityDistributions.f90:136-139)."""
        self.ctx.set_omega(omega)

    def ResetArea(self, on_off: bool = True) -> None:
        """ResetArea (:113-120). BVERK4 keeps areas frozen either way (:452, the stage area
        arrays of :66-71 are never read), so the flag is recorded only."""
        self.reset_areas = bool(on_off)

    # MPI setup (:126-230)
    def InitializeMPIRK4(self, aParticles: Particles, aPanels: Panels, procRank: int = 0,
                         numProcs: int = 1) -> None:
        self._mpi_ready = True
        self.LoadBalance(aParticles, aPanels, numProcs)

    def LoadBalance(self, aParticles: Particles, aPanels: Panels, numProcs: int = 1) -> dict:
        if not self._mpi_ready:
            raise RuntimeError("LoadBalance ERROR : MPI arrays not ready.")
        nA = aPanels.N_Active
        self._ranges = dict(particles=load_balance(aParticles.N, numProcs),
                            active=load_balance(nA, numProcs),
                            passive=load_balance(aPanels.N - nA, numProcs))
        return self._ranges

    def FinalizeMPIRK4(self) -> None:
        self.ResetRK4()
        self._mpi_ready = False
        self._ranges = None

    # Memory (:236-429)
    def ResetRK4(self) -> None:
        self._maps = None
        self.ctx.reset_rk4()

    # Time stepping
    def BVERK4(self, aParticles: Particles, aPanels: Panels, dt: float, procRank: int = 0,
               numProcs: int = 1) -> None:
        """One RK4 step of the barotropic vorticity equation on the whole grid
        (PanelVelocityParallel.f90:435-658). With numProcs > 1 use
        thesiscode_b200.dist.DistributedPanelVelocity, which splits targets by LoadBalance."""
        if numProcs != 1:
            raise ValueError("PanelVelocity runs one rank; use dist.DistributedPanelVelocity")
        if self._maps is None:  # InitRK4 + GatherPanels on the first call (:444-450)
            self._maps = gather_panels(aPanels)[0]
        maps, xA, zA, aA, xQ = gather_panels(aPanels, self._maps)
        xV = np.ascontiguousarray(aParticles.x)
        tke, ke = self.ctx.rk4_step(xA, zA, aA, xV, xQ, dt, 1)
        self.totalKE = float(tke[0])
        self.kineticEnergy = ke
        aParticles.x[:] = xV
        # :651 particles' relative vorticity follows the new latitude
        aParticles.relVort[:] = aParticles.absVort - 2.0 * self.ctx.get_omega() * aParticles.x[:, 2]
        if aPanels.tracer.shape[1] >= 2:  # :497-499, copied back by ScatterPanels
            aPanels.tracer[maps.active, 1] = ke
        scatter_panels(aPanels, maps, xA, zA, xQ)


    def StratosphereRK4(self, aParticles: Particles, aPanels: Panels, t: float, dt: float,
                        procRank: int = 0, numProcs: int = 1) -> None:
        """One forced RK4 step from time t (PanelVelocityParallel.f90:661-919): positions advance,
        the relative vorticity of panels and particles is rebuilt from absVort, the rotation and
        the Juckes forcing at t + dt (:908-915)."""
        if numProcs != 1:
            raise ValueError("PanelVelocity runs one rank")
        if self._maps is None:
            self._maps = gather_panels(aPanels)[0]
        maps, xA, _, aA, xQ = gather_panels(aPanels, self._maps)
        absA = np.ascontiguousarray(aPanels.absVort[maps.active])
        xV = np.ascontiguousarray(aParticles.x)
        relA, relV, tke, ke = self.ctx.strat_rk4_step(xA, absA, aA, xV, xQ, t, dt, 1,
                                                      absVortV=aParticles.absVort)
        self.totalKE = float(tke[0])
        self.kineticEnergy = ke
        aParticles.x[:] = xV
        aParticles.relVort[:] = relV
        if aPanels.tracer.shape[1] >= 2:
            aPanels.tracer[maps.active, 1] = ke
        scatter_panels(aPanels, maps, xA, relA, xQ)


_default: PanelVelocity | None = None


def _state() -> PanelVelocity:
    global _default
    if _default is None:
        _default = PanelVelocity()
    return _default


def BVERK4(aParticles, aPanels, dt, procRank=0, numProcs=1):
    _state().BVERK4(aParticles, aPanels, dt, procRank, numProcs)


def StratosphereRK4(aParticles, aPanels, t, dt, procRank=0, numProcs=1):
    _state().StratosphereRK4(aParticles, aPanels, t, dt, procRank, numProcs)


def InitializeMPIRK4(aParticles, aPanels, procRank=0, numProcs=1):
    _state().InitializeMPIRK4(aParticles, aPanels, procRank, numProcs)


def FinalizeMPIRK4():
    _state().FinalizeMPIRK4()


def LoadBalance(aParticles, aPanels, numProcs=1):
    return _state().LoadBalance(aParticles, aPanels, numProcs)


def ResetRK4():
    _state().ResetRK4()


def SetSmooth(new_smooth):
    _state().SetSmooth(new_smooth)


def GetSmooth():
    return _state().GetSmooth()


def ResetArea(on_off=True):
    _state().ResetArea(on_off)


def totalKE() -> float:
    return _state().totalKE


def kineticEnergy():
    return _state().kineticEnergy
