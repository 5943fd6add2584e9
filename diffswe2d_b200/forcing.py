"""Rainfall forcing for ``SWE2D`` (drop-in for ``RainfallForcing`` of the
reference's ``src/forcing.py``).

Rates already on the model grid, ``rates`` [nt,1,ny,nx] in m/s at ``times``
[nt] seconds; ``at(t)`` interpolates linearly in time and holds the first /
last record outside the series.  The interpolation is a PyTorch expression
evaluated once per step stage (off the kernels' path); it is written with the
same float operations as the reference's ``at`` so that a model forced by it
sees the reference's rain rates bit for bit.
"""
from __future__ import annotations

import torch
import torch.nn as nn


class RainfallForcing(nn.Module):
    def __init__(self, times: torch.Tensor, rates: torch.Tensor):
        super().__init__()
        if times.ndim != 1 or rates.ndim != 4 or rates.shape[0] != times.numel():
            raise ValueError("Expected times=[nt] and rates=[nt,1,ny,nx]")
        if times.numel() < 1:
            raise ValueError("Rainfall forcing needs at least one record")
        if times.numel() > 1 and not bool(torch.all(times[1:] > times[:-1])):
            raise ValueError("Rainfall times must be strictly increasing")
        self.register_buffer("times", times.clone())
        self.register_buffer("rates", rates.clone())

    def at(self, time) -> torch.Tensor:
        """Rain rate [1,1,ny,nx] at model time ``time`` (seconds)."""
        nt = self.times.numel()
        if nt == 1:
            return self.rates[0:1]
        t = torch.as_tensor(time, dtype=self.times.dtype, device=self.times.device)
        hi = torch.searchsorted(self.times, t).clamp(1, nt - 1)
        lo = hi - 1
        span = torch.clamp(self.times[hi] - self.times[lo], min=1.0e-12)
        w = (t - self.times[lo]) / span
        rate = (1.0 - w) * self.rates[lo] + w * self.rates[hi]
        rate = torch.where(t <= self.times[0], self.rates[0], rate)
        rate = torch.where(t >= self.times[-1], self.rates[-1], rate)
        return rate.unsqueeze(0)
