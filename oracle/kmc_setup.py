"""Oracle set-up for the kMC step: the FP64 oracle world that matches a GPU
replica (test infrastructure, used by the tests, smoke() and the bench's CPU
baseline only).

* ``rates`` -- the source and drain rates World::createSources /
  createDrains derive from the input keys (world.cpp:982-1030, 1110-1150).
* ``interface_bonds`` -- donor-acceptor bonds in the order
  lgm_kmc_set_morphology lists them.
* ``oracle_for`` -- a KmcOracle over a world's site energies, defects and
  carriers, with the same seed and replica key.
* ``independent_world`` -- the world a replica starts from, taken from the
  parameters alone: the library's host set-up (lgm_kmc_world_host), which
  tests/test_reference_pin.py pins bit for bit to the reference's own
  World::initialize; never read back from a GPU replica.
"""
import numpy as np


def rates(p):
    """World::createSources / createDrains (world.cpp:982-1030, 1110-1150)."""
    smart = lambda r, d: d if r < 0 else r
    if p.simulation_type == b"solarcell":
        gen = smart(p.generation_rate, p.source_rate)
        area = p.grid_x * p.grid_y
        if p.source_scale_area > 0 and p.source_scale_area != area:
            gen *= area / p.source_scale_area
        return dict(rate_e_source_l=smart(p.e_source_l_rate, 0.0),
                    rate_e_source_r=smart(p.e_source_r_rate, 0.0),
                    rate_h_source_l=smart(p.h_source_l_rate, 0.0),
                    rate_h_source_r=smart(p.h_source_r_rate, 0.0),
                    rate_e_drain_l=smart(p.e_drain_l_rate, p.drain_rate),
                    rate_e_drain_r=smart(p.e_drain_r_rate, p.drain_rate),
                    rate_h_drain_l=smart(p.h_drain_l_rate, p.drain_rate),
                    rate_h_drain_r=smart(p.h_drain_r_rate, p.drain_rate),
                    solar=1, generation_rate=gen, recombination_rate=p.recombination_rate,
                    recombination_range=p.recombination_range)
    return dict(rate_e_source_l=smart(p.e_source_l_rate, p.source_rate),
                rate_e_source_r=smart(p.e_source_r_rate, 0.0),
                rate_h_source_l=smart(p.h_source_l_rate, 0.0),
                rate_h_source_r=smart(p.h_source_r_rate, 0.0),
                rate_e_drain_l=smart(p.e_drain_l_rate, 0.0),
                rate_e_drain_r=smart(p.e_drain_r_rate, p.drain_rate),
                rate_h_drain_l=smart(p.h_drain_l_rate, 0.0),
                rate_h_drain_r=smart(p.h_drain_r_rate, 0.0))


def interface_bonds(phase, X, Y, Z):
    """Donor-acceptor bonds in the order lgm_kmc_set_morphology lists them:
    donor sites in increasing order, each with its acceptor neighbours at
    x-1, x+1, y-1, y+1, z-1, z+1."""
    ph = np.asarray(phase).reshape(Z, Y, X)
    s = np.arange(X * Y * Z, dtype=np.int64).reshape(Z, Y, X)
    nbr = np.full((Z, Y, X, 6), -1, np.int64)
    nbr[:, :, 1:, 0] = s[:, :, :-1]
    nbr[:, :, :-1, 1] = s[:, :, 1:]
    nbr[:, 1:, :, 2] = s[:, :-1, :]
    nbr[:, :-1, :, 3] = s[:, 1:, :]
    nbr[1:, :, :, 4] = s[:-1, :, :]
    nbr[:-1, :, :, 5] = s[1:, :, :]
    nbr = nbr.reshape(-1, 6)
    flat = ph.reshape(-1)
    ok = (nbr >= 0) & (flat[np.maximum(nbr, 0)] == 1) & (flat == 0)[:, None]
    src = np.broadcast_to(np.arange(X * Y * Z)[:, None], nbr.shape)
    return np.stack([src[ok], nbr[ok]], 1).reshape(-1).astype(np.int32)


def oracle_for(O, p, world, e, h, max_e, max_h, replica=0, step=0, phase=None):
    q = type(p).from_text("[Parameters]\n")  # fresh copy for the derived constants
    for name, _ in type(p)._fields_:
        setattr(q, name, getattr(p, name))
    q.check()
    orc = O.Oracle(q.grid_x, q.grid_y, q.grid_z, cutoff=q.electrostatic_cutoff,
                   hopping_range=q.hopping_range, sigma=q.coulomb_gaussian_sigma,
                   prefactor=q.electrostatic_prefactor)
    cfg = O.KmcConfig(inverse_kt=q.inverse_kt, exciton_binding=q.exciton_binding,
                      coulomb_carriers=q.coulomb_carriers, defects_charge=q.defects_charge,
                      image_terms=(2 if q.image_charges & 1 else 0) | (4 if q.image_charges & 2 else 0),
                      max_electrons=max_e, max_holes=max_h,
                      seed=q.random_seed & 0xFFFFFFFF, replica=replica,
                      source_metropolis=q.source_metropolis, source_coulomb=q.source_coulomb,
                      balance_charges=q.balance_charges, voltage_left=q.voltage_left,
                      voltage_right=q.voltage_right, **rates(q))
    bonds = None
    if phase is not None:
        cfg.confine = q.morphology_confine
        if q.generation_interface:
            bonds = interface_bonds(phase, q.grid_x, q.grid_y, q.grid_z)
    return O.KmcOracle(orc, world["site_energy"], world["defects"], e, h, cfg, step,
                       phase=phase, bonds=bonds)


def independent_world(p, replica=0):
    """Site energies, defects and seeded carriers of replica ``replica`` of
    parameters ``p`` (lgm_kmc_world_host, no device involved)."""
    from langmuir_b200.kmc import world_host
    return world_host(p, replica)


def assert_same_world(gpu_world, world):
    """The world a GPU replica holds equals the independent one."""
    np.testing.assert_array_equal(gpu_world["site_energy"], world["site_energy"])
    np.testing.assert_array_equal(gpu_world["defects"], world["defects"])
    np.testing.assert_array_equal(gpu_world["traps"], world["traps"])
    np.testing.assert_array_equal(gpu_world["trap_potentials"], world["trap_potentials"])
