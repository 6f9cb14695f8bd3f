"""Read-only GPU telemetry: SM clock and clock-event reasons sampled through
NVML in a background thread while a timed region runs.  Nothing here changes
any GPU setting."""
from __future__ import annotations

import statistics
import threading
import time

_REASONS = {
    "gpu_idle": "nvmlClocksEventReasonGpuIdle",
    "applications_clocks_setting": "nvmlClocksEventReasonApplicationsClocksSetting",
    "sw_power_cap": "nvmlClocksEventReasonSwPowerCap",
    "hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
    "sync_boost": "nvmlClocksEventReasonSyncBoost",
    "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
    "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
    "hw_power_brake_slowdown": "nvmlClocksEventReasonHwPowerBrakeSlowdown",
}


class ClockSampler:
    """Samples (sm_mhz, reasons bitmask, power W) every `period` seconds."""

    def __init__(self, device_index: int = 0, period: float = 0.005):
        self.period = period
        self.samples = []
        self._stop = threading.Event()
        self._thread = None
        self.ok = False
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.ok = True
        except Exception as exc:  # no NVML: report that, do not fail the run
            self.error = repr(exc)

    def _sample(self):
        nv = self.nv
        try:
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        except Exception:
            reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
        return (nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM), int(reasons),
                nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0)

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self._sample())
            except Exception:
                pass
            time.sleep(self.period)

    def start(self):
        if self.ok:
            self.samples = []
            self._stop.clear()
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def stop(self):
        if self._thread is not None:
            self._stop.set()
            self._thread.join()
            self._thread = None
            if self.ok:
                self.samples.append(self._sample())
        return self.summary()

    def summary(self) -> dict:
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": "NVML unavailable"}
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        mask = 0
        for _, r, _ in self.samples:
            mask |= r
        names = [name for name, attr in _REASONS.items() if mask & getattr(self.nv, attr, 0)]
        busy = [s for s in self.samples if not (s[1] & getattr(self.nv, _REASONS["gpu_idle"], 0))] or self.samples
        return {
            "sm_mhz": statistics.median(s[0] for s in busy),
            "sm_max_mhz": self.max_mhz,
            "reasons": names,
            "samples": len(self.samples),
            "power_w_max": max(s[2] for s in self.samples),
        }
