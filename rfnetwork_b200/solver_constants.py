"""Names shared by the setup API and the engine binding."""

# Key order of the coefficient dict built at rfnetwork/solver.py:1473-1518.
COEFF_NAMES = (
    "Ca_ex_y", "Ca_ex_z", "Cb_ex_y", "Cb_ex_z",
    "Ca_ey_z", "Ca_ey_x", "Cb_ey_z", "Cb_ey_x",
    "Ca_ez_x", "Ca_ez_y", "Cb_ez_x", "Cb_ez_y",
    "Da_hx_y", "Da_hx_z", "Db_hx_y1", "Db_hx_y2", "Db_hx_z1", "Db_hx_z2",
    "Da_hy_z", "Da_hy_x", "Db_hy_z1", "Db_hy_z2", "Db_hy_x1", "Db_hy_x2",
    "Da_hz_x", "Da_hz_y", "Db_hz_x1", "Db_hz_x2", "Db_hz_y1", "Db_hz_y2",
)

# Field codes of probes and monitors (rfnetwork/solver.py:1560).
FIELDS = ("ex", "ey", "ez", "hx", "hy", "hz")
