"""CPU: proposals built for all sources at once equal, byte for byte, the
reference's one-source-at-a-time construction (Galaxy.amplitudes,
damplitude_dsersic, damplitude_drh per source, forcepho/sources.py:607-694),
including the branches for sersic below the grid and rh < 0."""
import numpy as np


def test_vectorised_proposal_matches_per_source():
    from forcepho_b200.proposal import source_struct_dtype
    from forcepho_b200.sources import default_table, proposal_from_params
    tab = default_table()
    rng = np.random.default_rng(5)
    nb, ns = 3, 40
    params = np.zeros((ns, nb + 6))
    params[:, :nb] = rng.lognormal(0, 1, (ns, nb))
    params[:, nb:nb + 2] = rng.normal(0, 1e-4, (ns, 2))
    params[:, nb + 2] = rng.uniform(0.3, 1.0, ns)
    params[:, nb + 3] = rng.uniform(-1.5, 1.5, ns)
    params[:, nb + 4] = rng.uniform(0.5, 6.5, ns)        # some below the grid (0.8)
    params[:, nb + 5] = rng.uniform(-0.1, 1.2, ns)       # some rh < 0
    want = np.zeros(ns, dtype=source_struct_dtype)
    nr = tab.n_radii
    for i, p in enumerate(params):
        want["fluxes"][i, :nb] = p[:nb]
        ra, dec, q, pa, n, rh = p[nb:]
        want["ra"][i], want["dec"][i], want["q"][i], want["pa"][i] = ra, dec, q, pa
        want["nsersic"][i], want["rh"][i] = n, rh
        want["mixture_amplitudes"][i, :nr] = tab.amplitudes(n, rh)
        want["damplitude_drh"][i, :nr] = tab.damplitude_drh(n, rh)
        want["damplitude_dnsersic"][i, :nr] = tab.damplitude_dsersic(n, rh)
    got = proposal_from_params(params, nb, tab)
    assert np.any(params[:, nb + 4] < 0.8) and np.any(params[:, nb + 5] < 0)
    assert got.tobytes() == want.tobytes()
