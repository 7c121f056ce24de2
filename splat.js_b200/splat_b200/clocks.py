"""SM clock and clock-event reasons sampled during a timed region (read-only
NVML queries in a thread every 10 ms, else nvidia-smi every 200 ms), so a
measurement can show it ran at full clock with no thermal or hardware
slowdown."""
from __future__ import annotations

import statistics
import subprocess


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region: NVML
    in a thread every 10 ms (read-only queries), else nvidia-smi every 200 ms."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    # NVML clock-event reason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, device):
        self.device = device
        self.uuid = None
        self.p = None
        self.samples = []
        self.mx = None
        self.reasons = set()
        self._stop = None
        self._thread = None
        try:
            import torch
            self.uuid = "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
        except Exception:
            pass

    def _nvml_loop(self, handle, nv):
        import time as _t
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(handle, nv.NVML_CLOCK_SM)))
                try:
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(handle)
                except AttributeError:
                    bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(handle)
                for nm, b in self.REASON_BITS.items():
                    if bits & b:
                        self.reasons.add(nm)
            except Exception:
                pass
            _t.sleep(0.01)

    def __enter__(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            handle = nv.nvmlDeviceGetHandleByUUID(self.uuid) if self.uuid else nv.nvmlDeviceGetHandleByIndex(0)
            self.mx = float(nv.nvmlDeviceGetMaxClockInfo(handle, nv.NVML_CLOCK_SM))
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._nvml_loop, args=(handle, nv), daemon=True)
            self._thread.start()
            return self
        except Exception:
            self._thread = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.uuid or self.device)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self._thread:
            self._stop.set()
            self._thread.join(timeout=2)
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out, _ = self.p.communicate()

    def summary(self):
        sm, mx, reasons = list(self.samples), self.mx, set(self.reasons)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml 10 ms" if self.samples else "nvidia-smi 200 ms"}
