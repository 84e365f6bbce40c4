"""Bogacki-Shampine 3(2) time stepper on device tensors, restating scipy's
RK23 (scipy.integrate.RK23, scipy 1.18.1: scipy/integrate/_ivp/rk.py),
which the reference's quasidynamic Integrator drives (qd/integrator.py:44-54).

Same tableau, same error estimate (RMS norm of the embedded error over
atol + rtol max(|y|, |y_new|)), same step-size control (safety 0.9, factor
within [0.2, 10], no growth right after a rejection, minimum step 10 ulp of
t) and the same first-same-as-last reuse of the derivative, so the sequence
of accepted steps follows scipy's.  The state stays on the device; the one
host synchronisation per attempted step is the error norm (accept or
reject).  fun(t, y) -> dy/dt on tensors of y's device and dtype.
"""
import math

import numpy as np

SAFETY = 0.9
MIN_FACTOR = 0.2
MAX_FACTOR = 10.0

# Butcher tableau of RK23 (Bogacki & Shampine 1989)
C = (0.0, 1.0 / 2.0, 3.0 / 4.0)
A = ((), (1.0 / 2.0,), (0.0, 3.0 / 4.0))
B = (2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0)
E = (5.0 / 72.0, -1.0 / 12.0, -1.0 / 9.0, 1.0 / 8.0)
ERROR_EXPONENT = -1.0 / 3.0  # -1 / (error estimator order 2 + 1)


class RK23:
    def __init__(self, fun, t0, y0, t_bound, rtol=1e-3, atol=1e-6, first_step=None):
        self.fun = fun
        self.t = float(t0)
        self.y = y0.clone()
        self.t_bound = float(t_bound)
        self.direction = 1.0 if self.t_bound >= self.t else -1.0
        eps = np.finfo(np.float64).eps
        self.rtol = max(float(rtol), 100 * eps)
        self.atol = float(atol)
        self.n = y0.numel()
        self.f = fun(self.t, self.y)
        self.n_fun = 1
        if first_step is None:
            self.h_abs = self._initial_step()
        else:
            if first_step <= 0 or first_step > abs(self.t_bound - self.t):
                raise ValueError("first_step must be positive and within the bounds")
            self.h_abs = float(first_step)
        self.status = "running"
        self.n_rejected = 0

    def _rms(self, x):
        return float(x.norm()) / math.sqrt(self.n)

    def _initial_step(self):
        """scipy.integrate._ivp.common.select_initial_step (order 2)."""
        if self.n == 0:
            return math.inf
        scale = self.atol + self.y.abs() * self.rtol
        d0 = self._rms(self.y / scale)
        d1 = self._rms(self.f / scale)
        h0 = 1e-6 if d0 < 1e-5 or d1 < 1e-5 else 0.01 * d0 / d1
        h0 = min(h0, abs(self.t_bound - self.t))
        y1 = self.y + h0 * self.direction * self.f
        f1 = self.fun(self.t + h0 * self.direction, y1)
        self.n_fun += 1
        d2 = self._rms((f1 - self.f) / scale) / h0
        if d1 <= 1e-15 and d2 <= 1e-15:
            h1 = max(1e-6, h0 * 1e-3)
        else:
            h1 = (0.01 / max(d1, d2)) ** (1 / 3)
        return min(100 * h0, h1, abs(self.t_bound - self.t))

    def _rk_step(self, t, y, f, h):
        K0 = f
        K1 = self.fun(t + C[1] * h, y + (K0 * A[1][0]) * h)
        K2 = self.fun(t + C[2] * h, y + (K0 * A[2][0] + K1 * A[2][1]) * h)
        y_new = y + h * (K0 * B[0] + K1 * B[1] + K2 * B[2])
        f_new = self.fun(t + h, y_new)
        self.n_fun += 3
        err = (K0 * E[0] + K1 * E[1] + K2 * E[2] + f_new * E[3]) * h
        return y_new, f_new, err

    def step(self):
        """One accepted step (rejected attempts repeat with a smaller h);
        returns None like scipy's OdeSolver.step, or a failure message."""
        if self.status != "running":
            raise RuntimeError("attempt to step on a %s solver" % self.status)
        if self.n == 0 or self.t == self.t_bound:
            self.status = "finished"
            return None
        t, y = self.t, self.y
        min_step = 10 * abs(np.nextafter(t, self.direction * np.inf) - t)
        h_abs = min(max(self.h_abs, min_step), math.inf)
        step_rejected = False
        while True:
            if h_abs < min_step:
                self.status = "failed"
                return "Required step size is less than spacing between numbers."
            h = h_abs * self.direction
            t_new = t + h
            if self.direction * (t_new - self.t_bound) > 0:
                t_new = self.t_bound
            h = t_new - t
            h_abs = abs(h)
            y_new, f_new, err = self._rk_step(t, y, self.f, h)
            scale = self.atol + y.abs().maximum(y_new.abs()) * self.rtol
            error_norm = self._rms(err / scale)
            if error_norm < 1:
                if error_norm == 0:
                    factor = MAX_FACTOR
                else:
                    factor = min(MAX_FACTOR, SAFETY * error_norm ** ERROR_EXPONENT)
                if step_rejected:
                    factor = min(1.0, factor)
                h_abs *= factor
                break
            # rejected (an infinite or NaN norm shrinks by the minimum factor)
            shrink = SAFETY * error_norm ** ERROR_EXPONENT if error_norm == error_norm else 0.0
            h_abs *= max(MIN_FACTOR, shrink)
            step_rejected = True
            self.n_rejected += 1
        self.h_previous = h
        self.t_old = t
        self.t = t_new
        self.y = y_new
        self.h_abs = h_abs
        self.f = f_new
        if self.direction * (self.t - self.t_bound) >= 0:
            self.status = "finished"
        return None
