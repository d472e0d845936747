"""Temperature replica exchange over a batch of replicas on one GPU.

Restates the exchange controller of gromos-rs (crates/gromos-integrators/src/
remd.rs:168-420): replicas run ``exchange_interval`` MD steps (here all in
one batch, one CUDA graph launch per step, each with its own Berendsen bath,
berendsen_thermostat.rs:58-118), then neighbouring replicas on the
temperature ladder attempt an exchange with the Metropolis criterion
``delta = (beta_1 - beta_2) (E_2 - E_1)``, accepted when a uniform number is
below ``min(1, exp(-delta))`` (remd.rs:259-308).  Pairs follow the odd-even
scheme (remd.rs:211-226) or the sequential one.

An accepted exchange swaps the two replicas' temperatures instead of their
coordinates -- the same ensemble move without moving coordinates across the
device -- and rescales each replica's velocities to its new temperature
(replica.rs:355-371).  The random numbers come from a seeded generator, so
runs are reproducible (the reference draws from the thread RNG).

Across GPUs (one process per GPU, ``torch.distributed``): each rank passes
its own replicas with their global indices (``global_ids``) and the
temperatures of ALL replicas.  An attempt sums the potential energies over
the ranks with one all-reduce (a few bytes per replica), every rank then
takes the same seeded decisions over the whole ladder, and each rank applies
the temperature swaps of the replicas it holds.  No coordinates cross the
ranks, and the exchanges are those of one process holding every replica.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence

import numpy as np

from .nonbonded import Batch, Forcefield

KB = 0.00831446261815324  # kJ mol^-1 K^-1


class ReplicaExchange:
    def __init__(self, replicas: Sequence[Forcefield], temperatures: Sequence[float], exchange_interval: int = 100,
                 scheme: str = "odd_even", seed: int = 0, equilibration_steps: int = 0,
                 rescale_velocities: bool = True, batch: Optional[Batch] = None,
                 global_ids: Optional[Sequence[int]] = None, group=None):
        n_global = len(temperatures)
        if global_ids is None:
            global_ids = list(range(len(replicas)))
        if len(global_ids) != len(replicas) or len(set(global_ids)) != len(global_ids) or \
                any(not 0 <= int(g) < n_global for g in global_ids):
            raise ValueError("global_ids: one distinct index below len(temperatures) per local replica")
        if n_global < 2 or (group is None and not self._distributed(None) and len(replicas) != n_global):
            raise ValueError("need one temperature per replica and at least two replicas")
        if len({r.n_atoms for r in replicas}) > 1:
            raise ValueError("temperature exchange needs replicas of one system")
        if scheme not in ("odd_even", "sequential"):
            raise ValueError("scheme must be odd_even or sequential")
        self.replicas = list(replicas)
        self.global_ids = [int(g) for g in global_ids]
        self.local = {g: k for k, g in enumerate(self.global_ids)}   # global index -> local replica
        self.group = group
        self.n = n_global
        self.ladder = sorted(float(t) for t in temperatures)
        # position on the ladder of each (global) replica, and the replica at each position
        order = np.argsort(np.asarray(temperatures, dtype=float), kind="stable")
        self.at = [0] * n_global
        for pos, r in enumerate(order):
            self.at[int(r)] = pos
        self.interval = max(1, int(exchange_interval))
        self.scheme = scheme
        self.rng = np.random.default_rng(seed)
        self.equilibration = int(equilibration_steps)
        self.rescale = rescale_velocities
        self.odd_even_state = False
        self.step = 0
        self.attempts = np.zeros(n_global - 1, dtype=np.int64)
        self.accepts = np.zeros(n_global - 1, dtype=np.int64)
        self.own_batch = batch is None
        self.batch = batch or Batch()
        if self.own_batch:
            for r in self.replicas:
                self.batch.add(r)
        for r, g in zip(self.replicas, self.global_ids):
            r.md_set_temperature(self.ladder[self.at[g]], rescale_velocities=False)

    @staticmethod
    def _distributed(group) -> bool:
        import torch.distributed as dist
        return dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1

    def _energies(self) -> List[float]:
        """Potential energy (LJ + CRF) of every replica, indexed globally."""
        e = np.zeros(self.n, dtype=np.float64)
        for r, g in zip(self.replicas, self.global_ids):
            st = r.md_stats()
            e[g] = st["e_lj"] + st["e_crf"]
        if not self._distributed(self.group):
            return e.tolist()
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.from_numpy(e).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)   # each replica is held by one rank
        return t.cpu().tolist()

    def replica_at(self, pos: int) -> int:
        return self.at.index(pos)

    def temperature_of(self, replica: int) -> float:
        return self.ladder[self.at[replica]]

    def _pairs(self) -> List[tuple]:
        n = self.n
        if self.scheme == "sequential":
            start = 0
        else:
            start = 0 if self.odd_even_state else 1
            self.odd_even_state = not self.odd_even_state
        return [(p, p + 1) for p in range(start, n - 1, 2)]

    def attempt_exchanges(self) -> None:
        if self.step < self.equilibration:
            return
        energy = self._energies()
        for p, q in self._pairs():
            a, b = self.replica_at(p), self.replica_at(q)
            beta_a, beta_b = 1.0 / (KB * self.ladder[p]), 1.0 / (KB * self.ladder[q])
            delta = (beta_a - beta_b) * (energy[b] - energy[a])
            prob = 1.0 if delta < 0.0 else float(np.exp(-delta))
            accepted = self.rng.random() < prob
            self.attempts[p] += 1
            if accepted:
                self.accepts[p] += 1
                self.at[a], self.at[b] = q, p
                if a in self.local:
                    self.replicas[self.local[a]].md_set_temperature(self.ladder[q], rescale_velocities=self.rescale)
                if b in self.local:
                    self.replicas[self.local[b]].md_set_temperature(self.ladder[p], rescale_velocities=self.rescale)

    def run(self, total_steps: int) -> None:
        done = 0
        while done < total_steps:
            n = min(self.interval, total_steps - done)
            self.batch.md_run(n)
            done += n
            self.step += n
            if self.step % self.interval == 0:
                self.attempt_exchanges()

    def statistics(self) -> Dict:
        with np.errstate(divide="ignore", invalid="ignore"):
            rate = np.where(self.attempts > 0, self.accepts / np.maximum(self.attempts, 1), 0.0)
        return {"attempts": self.attempts.tolist(), "accepts": self.accepts.tolist(),
                "acceptance": rate.tolist(), "temperatures": [self.temperature_of(r) for r in range(self.n)]}

    def close(self) -> None:
        if self.own_batch:
            for r in self.replicas:
                self.batch.remove(r)
            self.batch.close()
