"""Physical constants (reference: physics/constant.py:17-41)."""

G = 9.81
P_0 = 1.01325e5
GAMMA = 1.4
W_AIR = 0.029
R_U = 8.314
R = R_U / W_AIR
CV = R / (GAMMA - 1.0)
CP = CV + R
KAPPA = R / CP
