"""Meson spectroscopy on the engine: the host side of observables/mesons.cpp:150-298 and
observables/propagator.cpp:10-19 over the device sources, propagator solves and
contractions of the C ABI (yg_create_*_source, yg_calc_propagator(_multi), yg_meson_contract).

``Mesons(lat, mass, prec, hits, method)`` is meson_init; ``measure()`` is meson_measure and
returns the correlators as the reference prints them (sign / (norm * hits), its channel
labels, including its print list's use of the g0g5g2 and g0g5g3 correlators for the labels
g0g5g1 and g0g5g2, mesons.cpp:293-295); ``lines()`` gives the printed text.  The random
source slice and the Z2 noise come from a numpy Generator (the reference's GSL stream is
not reproduced); explicit slices and noise may be passed instead."""
from __future__ import annotations

import numpy as np

SEMWALL, POINT = 0x01, 0x02          # include/spectrum.h:7-8

CHANNELS = ("id", "g1", "g2", "g3", "g5", "g5g1", "g5g2", "g5g3", "g0g1", "g0g2", "g0g3", "g0g5",
            "g0g5g1", "g0g5g2", "g0g5g3", "g5_g0g5")
# (printed label, correlator, sign), mesons.cpp:280-295
PRINT = (("id", "id", -1.0), ("g1", "g1", -1.0), ("g2", "g2", -1.0), ("g3", "g3", -1.0), ("g5", "g5", 1.0),
         ("g5g1", "g5g1", -1.0), ("g5g2", "g5g2", -1.0), ("g5g3", "g5g3", -1.0), ("g0g1", "g0g1", -1.0),
         ("g0g2", "g0g2", -1.0), ("g0g3", "g0g3", -1.0), ("g0g5", "g0g5", 1.0), ("g0g5g1", "g0g5g2", 1.0),
         ("g0g5g2", "g0g5g3", 1.0), ("g0g5g3", "g0g5g3", 1.0), ("g5_g0g5", "g5_g0g5", 1.0))

SQRT2INV = 0.70710678118654752440084436210


class Mesons:
    """meson_init(mass, prec, hits, method), mesons.cpp:150-209.  ``batched`` solves the
    propagators of a source slice together (yg_calc_propagator_multi, even-odd lattices, d = 3)
    instead of one auto_inverter call each, with ``solver`` "bicgstab" (default), "cg_mixed"
    or "cg"; ``mixed`` = True selects "cg_mixed"."""

    def __init__(self, lat, mass, prec, hits, method, rng=None, batched=False, mixed=False, solver=None):
        self.lat, self.mass, self.prec, self.hits = lat, mass, prec, int(hits)
        self.method = SEMWALL if method == SEMWALL else POINT
        self.T = lat.dims[0]
        self.vol3 = lat.V // self.T
        self.norm = self.vol3 if self.method == SEMWALL else 1
        self.ninv = 4 if self.method == SEMWALL else 4 * lat.d
        self.rng = rng if rng is not None else np.random.default_rng()
        self.batched = batched
        self.solver = solver or ("cg_mixed" if mixed else "bicgstab")
        self.source = lat.field()
        self.prop = [lat.field() for _ in range(self.ninv)]
        self.sources = [lat.field() for _ in range(self.ninv)] if batched else None
        self.raw = np.zeros((16, self.T))
        self.taus: list[int] = []
        self.iterations = 0

    def random_timeslice(self):
        """propagator.cpp:10-19: slice 1 with open or SF boundaries, else uniform"""
        if self.lat.bc in ("open", "sf"):
            return 1
        return int(self.rng.random() * self.T)

    def z2_noise(self):
        return np.where(self.rng.random(2 * self.lat.d * self.vol3) < 0.5, SQRT2INV, -SQRT2INV)

    def _solve_slice(self, tau, noise):
        lat = self.lat
        if not self.batched:
            for n in range(self.ninv):
                if self.method == SEMWALL:
                    lat.create_semwall_source(n, tau, self.source, noise if n == 0 else None)
                else:
                    lat.create_point_source(n, tau, self.source)
                self.iterations += lat.calc_propagator(self.mass, self.prec, self.prop[n], self.source)
            return
        for n in range(self.ninv):
            if self.method == SEMWALL:
                if n > 0:
                    lat.spinor_copy(self.sources[n], self.sources[n - 1])
                lat.create_semwall_source(n, tau, self.sources[n], noise if n == 0 else None)
            else:
                lat.create_point_source(n, tau, self.sources[n])
        for lo in range(0, self.ninv, 16):
            hi = min(lo + 16, self.ninv)
            its = lat.calc_propagator_multi(self.mass, self.prec, self.prop[lo:hi], self.sources[lo:hi],
                                            solver=self.solver)
            self.iterations += sum(its)

    def measure(self, taus=None, noises=None):
        """meson_measure, mesons.cpp:211-298: returns {label: printed values}"""
        self.raw[:] = 0
        self.taus = []
        for h in range(self.hits):
            tau = self.random_timeslice() if taus is None else int(taus[h])
            noise = None
            if self.method == SEMWALL:
                noise = self.z2_noise() if noises is None else noises[h]
            self.taus.append(tau)
            self._solve_slice(tau, noise)
            self.lat.meson_contract(self.method, tau, self.prop, self.raw)
        return self.values()

    def values(self):
        idx = {c: k for k, c in enumerate(CHANNELS)}
        sf = 1.0 / (self.norm * self.hits)
        return {lab: sign * sf * self.raw[idx[ch]] for lab, ch, sign in PRINT}

    def lines(self):
        """the MESONS lines of meson_measure: 'label: v0 v1 ...' with %1.6e values"""
        return [f"{lab}: " + "".join("%1.6e " % v for v in vals) for lab, vals in self.values().items()]
