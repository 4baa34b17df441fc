"""Seeded synthetic LTI workloads (numpy only, no device work).

A counter-based splitmix64 stream feeds uniforms on [0, 1) and Box-Muller
normals, so the same seed gives bit-identical systems in every process.  The
configurations are the benchmark and parity cases of this project:

  cfg1  RK4, n=8,   m=2,  p=2,  A = -2 I   + 0.5 G/sqrt(n), h=1e-3, T=4096
  cfg2  RK4, n=64,  m=8,  p=8,  A = -1.5 I + 0.5 G/sqrt(n), h=1e-4, T=2^20
  cfg3  ABM, n=128, m=16, p=16, A = -I     + 0.4 G/sqrt(n) (shifted so that
        max Re(lambda) <= -0.2), h=5e-4, T=2^18
  cfg4  4096 systems, n log-uniform in [4, 96], m = p = max(1, n//8),
        T log-uniform in [2^10, 2^16], RK4 for even ids, ABM for odd ids,
        A = -(1+U) I + 0.5 G/sqrt(n), h=1e-3

B, C, D and x0 are iid N(0,1); the input is u_j(t) = sum_{k<3} a_jk sin(2 pi
f_jk t + phi_jk) with a ~ U(0,1), f ~ U(0.1, 10), phi ~ U(0, 2 pi).  The
horizon end is t0 + (T - 1/2) h so that the step-count rule
floor((tEnd - t0)/h) + 1 gives exactly T outputs for both integrators.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


class Rng:
    """splitmix64 stream with vectorised draws."""

    def __init__(self, seed: int):
        self.state = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.count = 0

    def _u64(self, k: int) -> np.ndarray:
        idx = np.arange(self.count + 1, self.count + 1 + k, dtype=np.uint64)
        self.count += k
        with np.errstate(over="ignore"):
            z = self.state + idx * _GOLDEN
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
            z = z ^ (z >> np.uint64(31))
        return z

    def uniform(self, k: int) -> np.ndarray:
        return (self._u64(k) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)

    def normal(self, k: int) -> np.ndarray:
        pairs = (k + 1) // 2
        u = self.uniform(2 * pairs)
        u1 = 1.0 - u[0::2]
        u2 = u[1::2]
        r = np.sqrt(-2.0 * np.log(u1))
        z = np.empty(2 * pairs)
        z[0::2] = r * np.cos(2.0 * math.pi * u2)
        z[1::2] = r * np.sin(2.0 * math.pi * u2)
        return z[:k]


@dataclass
class Sinusoid:
    a: np.ndarray
    f: np.ndarray
    phi: np.ndarray

    @property
    def m(self) -> int:
        return self.a.shape[0]

    def __call__(self, t, i: int):
        return float(np.sum(self.a[i] * np.sin(2.0 * math.pi * self.f[i] * t + self.phi[i])))


@dataclass
class Case:
    name: str
    solver: int
    A: np.ndarray
    B: np.ndarray
    C: np.ndarray
    D: np.ndarray
    x0: np.ndarray
    u: Sinusoid
    h: float
    T: int
    t0: float = 0.0
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.A.shape[0]

    @property
    def m(self) -> int:
        return self.B.shape[1]

    @property
    def p(self) -> int:
        return self.C.shape[0]

    @property
    def t_end(self) -> float:
        return self.t0 + (self.T - 0.5) * self.h

    @property
    def scan_dim(self) -> int:
        return self.n if self.solver == 0 else 4 * self.n


def sinusoid(rng: Rng, m: int, K: int = 3) -> Sinusoid:
    a = rng.uniform(m * K).reshape(m, K)
    f = (0.1 + 9.9 * rng.uniform(m * K)).reshape(m, K)
    phi = (2.0 * math.pi * rng.uniform(m * K)).reshape(m, K)
    return Sinusoid(a, f, phi)


def lti(rng: Rng, name: str, solver: int, n: int, m: int, p: int, diag: float, scale: float, h: float, T: int,
        max_re: Optional[float] = None) -> Case:
    G = rng.normal(n * n).reshape(n, n)
    A = diag * np.eye(n) + scale * G / math.sqrt(n)
    if max_re is not None:
        lam = float(np.max(np.linalg.eigvals(A).real))
        if lam > max_re:
            A = A - (lam - max_re) * np.eye(n)
    B = rng.normal(n * m).reshape(n, m)
    C = rng.normal(p * n).reshape(p, n)
    D = rng.normal(p * m).reshape(p, m)
    x0 = rng.normal(n)
    u = sinusoid(rng, m)
    return Case(name, solver, A, B, C, D, x0, u, h, T)


def cfg1() -> Case:
    return lti(Rng(1235), "cfg1", 0, 8, 2, 2, -2.0, 0.5, 1e-3, 4096)


def cfg2(T: int = 1 << 20) -> Case:
    return lti(Rng(1236), "cfg2", 0, 64, 8, 8, -1.5, 0.5, 1e-4, T)


def cfg3(T: int = 1 << 18) -> Case:
    return lti(Rng(1237), "cfg3", 1, 128, 16, 16, -1.0, 0.4, 5e-4, T, max_re=-0.2)


def cfg4(count: int = 4096, seed: int = 1238) -> List[Case]:
    rng = Rng(seed)
    cases = []
    for i in range(count):
        n = int(round(math.exp(math.log(4) + (math.log(96) - math.log(4)) * float(rng.uniform(1)[0]))))
        T = int(round(math.exp(math.log(2 ** 10) + (math.log(2 ** 16) - math.log(2 ** 10)) * float(rng.uniform(1)[0]))))
        m = p = max(1, n // 8)
        diag = -(1.0 + float(rng.uniform(1)[0]))
        cases.append(lti(rng, f"cfg4[{i}]", i % 2, n, m, p, diag, 0.5, 1e-3, T))
    return cases


def cfg5(count: int, rate: float, seed: int = 1239, n_range=(8, 256), T_range=(1e3, 1e6)):
    """Serving workload: `count` requests with Poisson arrivals at `rate` per
    second; n and T log-uniform in the given ranges, RK4 / ABM 50/50,
    m = p = max(1, n/8), A = -(1+U(0,1)) I + 0.5 G/sqrt(n), h = 1e-3.
    Returns [(arrival_s, Case)]."""
    rng = Rng(seed)
    out = []
    t = 0.0
    for i in range(count):
        t += -math.log(max(1e-300, 1.0 - float(rng.uniform(1)[0]))) / rate
        n = int(round(math.exp(math.log(n_range[0]) + (math.log(n_range[1]) - math.log(n_range[0])) *
                               float(rng.uniform(1)[0]))))
        T = int(round(math.exp(math.log(T_range[0]) + (math.log(T_range[1]) - math.log(T_range[0])) *
                               float(rng.uniform(1)[0]))))
        T = max(T, 5)
        m = p = max(1, n // 8)
        solver = 0 if float(rng.uniform(1)[0]) < 0.5 else 1
        diag = -(1.0 + float(rng.uniform(1)[0]))
        out.append((t, lti(rng, f"cfg5[{i}]", solver, n, m, p, diag, 0.5, 1e-3, T)))
    return out


def small(seed: int, solver: int, n: int, m: int, p: int, T: int, h: float = 1e-2, diag: float = -1.0,
          scale: float = 0.5) -> Case:
    """A small random stable case for parity sweeps."""
    return lti(Rng(seed), f"small{seed}", solver, n, m, p, diag, scale, h, T)
