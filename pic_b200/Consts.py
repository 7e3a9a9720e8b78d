"""Physical constants with the reference's values (src/Consts.py:1-11).

qe is 1.6e-19 as in the reference (not the CODATA value) so that the oracle
and this build agree; AMU is the 1.66e-27 kg used by the reference's inputs
(test.inp:79).
"""
qe = 1.6e-19
qe_1 = 1 / qe
me = 9.10938356e-31
mp = 1.67262158e-27
eps0 = 8.85418782e-12
eps0_sqrt = eps0 ** 0.5
eps0_1 = 1 / eps0
mu0 = 1.25663706e-6
kb = 1.380649e-23
c = 2.99792458e8
e_p_ratio = mp / me
AMU = 1.66e-27
