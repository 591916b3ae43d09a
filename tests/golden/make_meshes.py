"""Copy the reference's two test meshes into tests/golden/ as fixtures.

    EMUSTACK_REF=<path to the EMUstack tree> python tests/golden/make_meshes.py

backend/fortran/msh/4testing-600_120.mail (1 077 nodes, 518 P2 triangles)
and 4testing-940_266_sq.mail (5 121 nodes, 2 528 triangles) are the meshes
the reference's own tests solve on.  They are copied byte for byte, so the
overlap tests read them with ``emustack_b200.mesh.Mesh.from_mail`` exactly as
the reference's mesh reader (backend/fortran/geometry.f:27-60) would; nothing
at test time reads the reference tree.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ('4testing-600_120.mail', '4testing-940_266_sq.mail')


def main():
    ref = os.environ.get('EMUSTACK_REF')
    if not ref or not os.path.isdir(os.path.join(ref, 'backend', 'fortran', 'msh')):
        raise SystemExit('set EMUSTACK_REF to the root of the EMUstack source tree')
    for nm in NAMES:
        shutil.copyfile(os.path.join(ref, 'backend', 'fortran', 'msh', nm), os.path.join(HERE, nm))
        print('copied', nm)


if __name__ == '__main__':
    sys.exit(main())
