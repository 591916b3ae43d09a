"""Generate tests/golden/materials.npz from the EMUstack reference: the
refractive indices its own Material.n (backend/materials.py:131-161) returns
for a constant index, synthetic tables of (wavelength, n) and (wavelength,
Re n, Im n) rows and Drude parameters, at wavelengths that include the
table nodes and both ends, with Anallo.n's loss flag
(backend/mode_calcs.py:186-192) applied as np.real.

    EMUSTACK_REF=<path to the EMUstack tree> python tests/golden/make_materials_golden.py

The reference is imported as tests/golden/make_golden.py imports it.  The
tables are synthetic (seeded), not the reference's data files.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main():
    import make_golden
    objects, materials, stack, mode_calcs = make_golden.import_reference()
    rng = np.random.default_rng(20261204)
    wl = np.sort(rng.uniform(300, 1200, 41))
    wl[0], wl[-1] = 300.0, 1200.0
    complex_tab = np.stack([wl, 1.5 + rng.uniform(0, 2.5, 41), rng.uniform(0, 0.6, 41)], axis=1)
    real_tab = np.stack([np.append(wl[:-2:2], 1200.0), 1.3 + rng.uniform(0, 1, 21)], axis=1)
    drude = np.array([1.36e16, 1.05e14, 9.5])
    specs = {'const': np.array(2.1 + 0.03j), 'complex_tab': complex_tab, 'real_tab': real_tab, 'drude': drude}
    q = np.concatenate([rng.uniform(300, 1200, 200), complex_tab[:, 0], real_tab[:, 0], [300.0, 1200.0]])
    d = {'wl': q}
    for name, spec in specs.items():
        d['spec_' + name] = spec
        try:
            m = materials.Material(spec.item() if spec.shape == () else spec)
            n = np.array([complex(np.asarray(m.n(w)).item()) for w in q])
        except Exception as e:   # the reference cannot build this kind under numpy 2
            print('skipped', name, repr(e))
            continue
        d['n_' + name] = n
    out = os.path.join(HERE, 'materials.npz')
    np.savez_compressed(out, **d)
    print('wrote', out, sorted(d))


if __name__ == '__main__':
    main()
