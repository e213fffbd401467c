"""A bla.i written by the tests, in the record order of bla/rparambl.f
(version 20070716): the temporal channel with the values the tests vary."""


def bla_i(namnin="init.u", namnut="end.u", tmax=0.0, maxit=0, dt=0.0, nst=4, cflmaxin=0.8, xl=12.566,
          cflux=True, retau=180.0, sgs=False, icfl=4, iamp=0, namamp="amp.stat", ixys=0, saves=(),
          spat=False, rbfl=None, fringe=(1.0, -13.0, 0.0, 7.0, 3.0), ampob=0.0):
    """spat: a spatial run with the fringe (fmax, fstart, fend, frise, ffall)
    and the base flow read from the file rbfl (None: computed)."""
    rec = ["# bla.i written by the tests", "20070716        Version of input file", namnin, namnut,
           f"{tmax}            Maximum simulation time (tmax)", f"{maxit}   Maximum iterations (maxit)",
           "-200            Maximum CPU time (cpumax)", "-200            Maximum wall-clock time (wallmax)",
           ".false.          Save intermediate files (write_inter)", f"{dt}   Time step (dt)",
           f"{nst}   number of RK stages (nst)", f"{cflmaxin}   CFL number (cflmaxin)", f"{xl}  Box length (xl)",
           ".true.         Variable size (varsiz)", ".0              Rotation rate (rot)",
           (".true." if cflux else ".false.") + "          Constant mass flux (cflux)"]
    if not cflux:
        rec.append(f"{retau}    Re_tau")
    rec += [".false.         Perturbation mode (pert)", "0               Boundary condition number (ibc)",
            ".false.         Chebyshev integration method (cim)", ".false.         Galilei transformation (gall)",
            ".false.         Constant wall-suction (suction)",
            (".true." if spat else ".false.") + "         Spatial simulation (spat)"]
    if spat:
        rec += [".false.         Tabulated free-stream velocity (tabfre)",
                (".true." if rbfl else ".false.") + "         Read base flow from file (rbfl)"]
        if rbfl:
            rec.append(rbfl)
        rec += [f"{v}   {name}" for v, name in zip(fringe, ("Fringe strength (fmax)", "Fringe start (fstart)",
                                                          "Fringe end (fend)", "Fringe rise distance (frise)",
                                                          "Fringe fall distance (ffall)"))]
        rec += [f"{ampob}             Amplitude oblique waves (ampob)", "0.0             Amplitude 2D TS waves (amp2d)",
                ".false.         Forcing with Orr-Sommerfeld modes (osmod)",
                ".false.         Forcing with streaks (streak)", ".false.         Forcing with waves (waves)"]
    else:
        rec.append("0.              Temporal development vel. (cdev)")
    rec += [(".true." if sgs else ".false.") + "         Read sgs.i (sgs)", "0               SFD (isfd)",
            "0               MHD (imhd)", "0               Type of localized disturbance (loctyp)",
            ".false.         Trip forcing (tripf)", "0               Boundary condition at lower wall (wbci)",
            f"{icfl}              CFL calculation interval (icfl)",
            f"{iamp}    Amplitude calculation interval (iamp)"]
    if iamp > 0:
        rec += [namamp, ".false."]
    rec += [".false.         y-dependent statistics (longli)",
            "0               Extremum calculation interval (iext)",
            f"{ixys}              xy-statistics calculation interval (ixys)"]
    if ixys > 0:
        rec += ["xy.stat", "64              xy-statistics saving interval (ixyss)", "200.  Start time (txys)",
                ".false.         Two-point correlations in z (corrf)",
                ".false.         Two-point correlations in x (corrf_x)", ".false.         Time series (serf)"]
    rec.append(f"{len(saves)}               Number of 3D fields to save (msave)")
    for t, name in saves:
        rec += [f"{t}", name]
    rec += ["0               Number of wavenumbers to save (mwave)",
            "0               Number of planes to save (npl)"]
    return "\n".join(rec) + "\n"
