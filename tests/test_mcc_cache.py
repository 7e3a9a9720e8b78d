"""The operator cache of null_collision_method (host logic, no GPU).

Operators are keyed by the contents of the cross-section tables, not by the
identity of the table objects: a garbage-collected table's id can be reused
by a new object with other values, which must never get the old operator."""
from types import SimpleNamespace

import numpy as np

from pic_b200 import MCC


def particles(*masses):
    return SimpleNamespace(species=[SimpleNamespace(mass=m, charge=q, collision_model=c) for m, q, c in masses])


def key(p, xs, **kw):
    args = dict(density=1e21, dt=1e-11, ionization=True, seed=0, gas_temperature=300.0, gas_mass=6.6e-26,
                threshold=15.6)
    args.update(kw)
    return MCC._operator_key(p, args["density"], xs, args["dt"], args["ionization"], args["seed"],
                             args["gas_temperature"], args["gas_mass"], args["threshold"])


def test_key_follows_table_contents():
    p = particles((9.1e-31, -1.6e-19, 0), (6.6e-26, 1.6e-19, 1))
    E = np.geomspace(0.01, 1000, 50)
    a = ((E, 1e-19 / (1 + E)), (E, np.where(E > 15.8, 3e-20, 0.0)))
    b = ((E.copy(), (1e-19 / (1 + E)).copy()), (E.copy(), np.where(E > 15.8, 3e-20, 0.0)))
    assert key(p, a) == key(p, b)  # other objects, same values
    c = ((E, 1e-19 / (1 + E)), (E, np.where(E > 15.8, 3.0000001e-20, 0.0)))
    assert key(p, a) != key(p, c)  # one value differs
    assert key(p, a) != key(p, ((E, 1e-19 / (1 + E)), (None, None)))
    assert key(p, a) != key(p, a, seed=1)
    assert key(p, a) != key(p, a, dt=2e-11)
    assert key(p, a) != key(particles((9.1e-31, -1.6e-19, 0)), a)
    # the split between columns is part of the key
    assert key(p, ((E[:10], E[10:]),)) != key(p, ((E[:20], E[20:]),))
