"""emustack_b200: B200-native generalised scattering-matrix (GSM) stage of EMUstack.

Drop-in objects (same names and attributes as the reference's backend):

    from emustack_b200 import objects, materials
    from emustack_b200.stack import Stack

Batched GPU entry points: ``emustack_b200.films.FilmStackSolver`` (all-film
stacks, one launch per batch).  Every numeric path runs CUDA kernels from
libemustack_gsm.so (built by ``emustack_b200.build.build_library``); there is
no CPU fallback.
"""
__version__ = '0.1.0'
