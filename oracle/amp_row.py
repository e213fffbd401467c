"""The amp.stat line of the reference for the channel (fltype = 1), restated
in numpy from the plane statistics amp(nyp,20).

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the row that the
library's sgpu_amplitudes computes on the host from its device statistics.

Follows bla/wampbl.f:124-278 with dstar = 1 and one process (no MPI gather):
amp(y,8) is negated and amp(y,13) = amp(y,9) (:184-185), sums 1..10 and 13
are Clenshaw-Curtis integrals with wint (:190-203; bla/preprbl.f:78-87), the
99 % / displacement / momentum thicknesses use gridy = 1 + eta
(bla/preprbl.f:56-58, wampbl.f:209-227), sums 1..7 become rms values
sqrt(sum/2) (:232-234), wb = sum10/2, e0 = sqrt((sum9 + sum10)/2),
tau1 = amp(1,12), tau2 = amp(nyp,12), h+ = sqrt((|tau1| + |tau2|) Re / 2)
(:238-246), and the written row is (:276-278)
  t, sum1..3, sum4..6, sum7, sum8, e0, h+, px, sum13 Re / 2, tau1, tau2,
  delta1..3, wb.
"""
import numpy as np


def wint_gridy(nyp):
    pi = 3.1415926535897932385
    wint = np.empty(nyp)
    for y in range(nyp):
        w = -.5
        for i in range(1, (nyp + 1) // 2 - 1):
            w = w + np.cos(pi * float(2 * i * y) / float(nyp - 1)) / float((2 * i) ** 2 - 1)
        w = w + .5 * np.cos(pi * float(y)) / float((nyp - 1) ** 2 - 1)
        w = -4. / float(nyp - 1) * w
        if y in (0, nyp - 1):
            w = w * .5
        wint[y] = w
    gridy = np.array([1. + np.cos(pi * float(y) / float(nyp - 1)) for y in range(nyp)])
    return wint, gridy


def amp_row(amp, t, re, px):
    """amp: array (20, nyp), amp[k-1, y-1] = amp(y, k).  Returns the 19 values."""
    a = np.array(amp, dtype=np.float64, copy=True)
    nyp = a.shape[1]
    wint, gridy = wint_gridy(nyp)
    a[7] = -a[7]
    a[12] = a[8]
    s = np.zeros(21)
    for i in list(range(1, 11)) + [13]:
        acc = 0.0
        for y in range(nyp):
            acc = acc + a[i - 1, y] * wint[y]
        s[i] = acc
    d = [0.0, 0.0, 0.0, 0.0]
    u = a[12]
    for y in range(nyp):
        if d[1] == 0. and u[y] <= 0.99:
            if u[y] == 0.99 or y == 0:
                d[1] = gridy[y]
            else:
                d[1] = gridy[y] + (0.99 - u[y]) * (gridy[y - 1] - gridy[y]) / (u[y - 1] - u[y])
        d[2] = d[2] + (1. - u[y]) * wint[y]
        d[3] = d[3] + u[y] * (1. - u[y]) * wint[y]
    for j in range(1, 8):
        s[j] = np.sqrt(s[j] * .5)
    wb = s[10] * .5
    e0 = np.sqrt((s[9] + s[10]) * .5)
    tau1, tau2 = a[11, 0], a[11, nyp - 1]
    hplus = np.sqrt((abs(tau1) + abs(tau2)) * re / 2.)
    return np.array([t, s[1], s[2], s[3], s[4], s[5], s[6], s[7], s[8], e0, hplus, px, s[13] * re / 2.,
                     tau1, tau2, d[1], d[2], d[3], wb])
