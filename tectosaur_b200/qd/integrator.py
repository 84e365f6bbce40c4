"""Time integration of a quasidynamic model (reference:
tectosaur/qd/integrator.py:8-75): RK23 with atol = rtol = timestep_tol,
started at init_step_size, the state kept on the device."""
from . import siay
from .rk23 import RK23


class Integrator:
    def __init__(self, model, init_conditions, init_step_size=siay / 10.0):
        from ..util import device
        self.model = model
        self.derivs = model.make_derivs()
        t0, y0 = init_conditions
        if not device.is_device_tensor(y0):
            y0 = device.to_dev(y0)
        self.init_conditions = (t0, y0)
        self.h_t = []
        self.h_y = []
        tol = model.cfg["timestep_tol"]
        self.rk23 = RK23(self.derivs, t0, y0, 1e50, rtol=tol, atol=tol,
                         first_step=init_step_size)

    def step_idx(self):
        return len(self.h_t)

    def integrate(self, n_steps, until=None, display_fnc=None, display_interval=1):
        """n_steps accepted steps (or until t passes `until`); each step's
        (t, y) is appended to h_t / h_y (y stays a device tensor)."""
        for i in range(n_steps):
            if until is not None and self.rk23.t > until:
                return
            msg = self.rk23.step()
            if msg is not None:
                raise RuntimeError("time step failed: " + msg)
            self.h_t.append(self.rk23.t)
            self.h_y.append(self.rk23.y)
            if display_fnc is not None and i % display_interval == 0:
                display_fnc(self)
