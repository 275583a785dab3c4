"""CPU oracle for the Ves3D StokesVelocity path -- TEST INFRASTRUCTURE ONLY.

Restates the reference's algorithm (lu1and10/ves3d) on the CPU so that the CUDA path
can be checked against it. Only tests/, bench.py's cpu_baseline / reference leg and
__graft_entry__.smoke() may import anything from here, and only as the checker or the
timed CPU baseline -- never as the thing measured or shipped.

  sh.py      numpy restatement of SphericalHarmonics (transforms, rotations, singular
             quadrature, self matrix)
  direct.c   C restatement of StokesAlltoAll / DirectStokesKernel
  stokes.py  the FP64 StokesVelocity composition
  reflib.py  loader for oracle/_ref/, the reference's own CPU code compiled in place
             by oracle/ref/Makefile (used to pin the restatement)
"""
