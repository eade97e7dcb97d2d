"""Oracle constants: the unit factors of ``src/Kappa/Src/constants.f90:27-71``.

Test infrastructure only.  Same literal expressions as the reference so that
products of prefactors agree to the last bit with the reference's FP64 values.
"""
import math

PI = 4.0 * math.atan(1.0)
Onebysqrt2PI = 1.0 / math.sqrt(2.0 * PI)
cmp_prec = 1.0e-8
zero_prec = 5.0e-5
OnebySix = 0.16666666666666666
# ``EPS = 1.0E-8`` is a default-real (single precision) literal in the reference, widened to dp
EPS = float(__import__("numpy").float32(1.0e-8))
wTHz = math.sqrt(1.60217733 * 6.02214076 * 10.0) * 10.0
THzConv = wTHz / (2.0 * PI)
vg_ms = wTHz * 100.0
BEConv = math.sqrt(1.60217733 * 6.02214076 * 10.0) * 6.582119569 * 100.0 / 8.617333262
Sctr3THz2 = 1.054571817 * (1.60217733 ** 2) * (6.02214076 ** 3) * 1000000.0 * PI * 0.0625
Sctr4THz2 = 0.125 * PI * ((1.054571817 * 1.602176565) ** 2) * (6.022140857 ** 4) * 1000000.0
kW_m_k = (1.054571817 ** 2) * 0.001 / 1.380649
# kappa_iter constants (src/Kappa/Src_iterative/constants.f90:53-58): pi/4 prefactor
Sctr3THz2_iter = 1.054571817 * (1.60217733 ** 2) * (6.02214076 ** 3) * 1000000.0 * PI * 0.25
