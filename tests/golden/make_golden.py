"""Regenerates the oracle's own golden trajectories (self-made fixtures).

Run from the repository root:  python tests/golden/make_golden.py
The UEG fixture is not generated: its numbers are the reference's expected
output (see its 'source' field).
"""
import json
import os
import sys
import warnings

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
warnings.simplefilter("ignore")

from oracle import coupled_cluster, inputs, triples  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def c0():
    opts = dict(method="Ccsd", maxIterations=40, energyConvergence=1e-10,
                amplitudesConvergence=1e-6, mixer=dict(type="DiisMixer", maxResidua=5))
    s = inputs.config_system("c0", seed=0)
    r = coupled_cluster.run(s, **opts)
    T1, T2 = r["amplitudes"]
    out = dict(source="oracle (self-made golden)", config="c0", seed=0, options=opts,
               iterations=r["iterations"], converged=bool(r["convergenceReached"]),
               energy=r["energy"],
               history_energy=[h["energy"] for h in r["history"]],
               history_dR=[h["dR"] for h in r["history"]],
               T1_norm=float((T1 ** 2).sum() ** 0.5), T2_norm=float((T2 ** 2).sum() ** 0.5))
    # (T) at the converged amplitudes (tuple-loop restatement; the full-array
    # restatement agrees on the smaller systems of the tests)
    V = triples.triples_integrals(s)
    out["triples"] = dict(correlation=triples.triples_atrip(T1, T2, V, s.eps_h, s.eps_p))
    json.dump(out, open(os.path.join(HERE, "c0_seed0.json"), "w"), indent=1)


if __name__ == "__main__":
    c0()
