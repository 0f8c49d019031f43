"""CPU oracle for the litepgo volumetric neo-Hookean hot path.

TEST INFRASTRUCTURE ONLY: a plain C++17 restatement of the reference CPU path
(see lpg_oracle.cpp for the file:line citations), loaded through ctypes. Only
tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
may import it. The product package (litepgo_b200) never does.
"""

from .oracle import (  # noqa: F401
    DOMAIN_ERROR,
    HEX_CORNERS,
    INVALID_ARGUMENT,
    LOGIC_ERROR,
    OracleError,
    hex_box,
    hex_dN_dxi,
    hex_eval,
    hex_force_vjp_theta,
    hex_hermite_eval,
    hex_hermite_force_vjp_theta,
    hex_hermite_N_dN,
    hermite_box,
    hex_points,
    OracleMesh,
    build,
    lib,
    nh_W,
    nh_dW_dF,
    nh_d2W_dF2,
    nh_d2W_dF_dtheta,
    nh_d2W_dF_dFp,
    nh_feasible_step,
    positive_det_step,
    project_psd,
    set_threads,
    get_threads,
)
