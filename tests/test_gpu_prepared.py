"""PreparedSimulationTest (vexelray-sim-fluid-gui/src/test/java/dev/vexelray/sim/fluid/gui/PreparedSimulationTest.java):
a 3D simulation made in two halves on two threads. The slow half (vf_mpm3_prepare: every allocation, nothing
submitted) runs on a worker while the owning thread goes on stepping the simulation already running; the rest
(vf_mpm3_create: clearing the buffers) runs on the owning thread. It starts empty, as one made in one go does, and
conserves the water's mass. Bars: the reference's, the grid's mass within 1e-4 of the particles', every node finite.
"""
import math
import threading

import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, WALL, JavaRandom, stable_step

pytestmark = pytest.mark.gpu

N, PPC, RHO0 = 32, 8, 1.0
G = 9.81 * (N - 1)


def column(cols, rows, layers):
    """PreparedSimulationTest.Dam.column (PreparedSimulationTest.java:103-123): seed 1, eight particles a cell."""
    count = cols * rows * layers * PPC
    at = np.empty((3, count), F)
    r = JavaRandom(1)
    k = 0
    for layer in range(layers):
        for row in range(rows):
            for col in range(cols):
                for _ in range(PPC):
                    at[0, k] = (WALL + F(col)) + r.next_float() * F(0.999)
                    at[1, k] = (WALL + F(row)) + r.next_float() * F(0.999)
                    at[2, k] = (WALL + F(layer)) + r.next_float() * F(0.999)
                    k += 1
    mass = np.full(count, F(RHO0 / PPC), F)
    fall = math.sqrt(2 * G * rows)
    bulk = 25 * fall * fall * RHO0
    dt = stable_step(bulk, RHO0, 2.5 * fall, 0.45 * 2 / 3)
    return at, mass, vf.flip3_params(dt, 0, -G, 0, bulk, RHO0)


def assert_mass(mass, grid_mass):
    assert np.all(np.isfinite(grid_mass)), "a broken node"
    expected = float(mass.astype(np.float64).sum())
    assert abs(float(grid_mass.astype(np.float64).sum()) - expected) <= expected * 1e-4, "the grid holds the mass"


def test_a_simulation_prepared_on_a_worker_starts_empty_and_steps_on_the_owning_thread():
    running = column(8, 12, 8)
    nxt = column(10, 16, 10)
    box = {}

    def prepare():
        box["prepared"] = vf.ParticleSimulation3.prepare(N, N, N, nxt[0].shape[1])

    with vf.ParticleSimulation3(N, N, N, running[0].shape[1]) as live:
        assert live.on_gpu()
        live.load(list(running[0]), [np.zeros(running[0].shape[1], F)] * 3, running[1], running[2])
        worker = threading.Thread(target=prepare)
        worker.start()
        steps = 0
        while True:   # the owning thread steps the running simulation while the worker prepares the next
            live.advance(1)
            live.finish()
            steps += 1
            if not worker.is_alive():
                break
        worker.join()
        assert steps > 0
        assert_mass(running[1], live.grid()[0])
        prepared = box["prepared"]
        with vf.ParticleSimulation3(prepared) as sim:
            assert sim.on_gpu()
            assert sim.particles() == nxt[0].shape[1]
            assert np.all(sim.grid()[0] == 0.0), "cleared, as one made in one go starts"
            sim.load(list(nxt[0]), [np.zeros(nxt[0].shape[1], F)] * 3, nxt[1], nxt[2])
            sim.advance(200)
            assert_mass(nxt[1], sim.grid()[0])
        with pytest.raises(vf.IllegalStateException):
            vf.ParticleSimulation3(prepared)


def test_a_preparation_never_started_is_freed_by_closing_it():
    box = {}
    worker = threading.Thread(target=lambda: box.setdefault("p", vf.ParticleSimulation3.prepare(N, N, N, 64)))
    worker.start()
    worker.join()
    prepared = box["p"]
    prepared.close()
    prepared.close()
    with pytest.raises(vf.IllegalStateException):
        vf.ParticleSimulation3(prepared)
