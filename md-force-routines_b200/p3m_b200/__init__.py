"""p3m_b200: B200-native P3M force step and integrator for Yukawa OCP MD.

The reference-named modules next to this package (yukawa_pp, yukawa_pm_ord6,
yukawa_gf_opt, yukawa_p3m_ord6, velocity_verlet_p3m_ord6,
thermostat_p3m_ord6, initialize_pos_vel, s_of_q_w, s_of_q_w_avg) keep the reference's call
signatures and route every stage through libp3m_b200.so.
"""
from ._lib import FP32, FP64, MODE_NVE, MODE_THERMOSTAT, P3MError, lib  # noqa: F401
from .context import (Context, Replica, compat_context, compat_precision,  # noqa: F401
                      fp32_peak_tflops, gf_opt_device, set_compat_precision, sqw_runs,
                      sqw_series)

__all__ = ["Context", "Replica", "P3MError", "FP32", "FP64", "MODE_NVE", "MODE_THERMOSTAT",
           "compat_context", "set_compat_precision", "compat_precision", "gf_opt_device",
           "fp32_peak_tflops", "sqw_series", "sqw_runs", "lib"]
