"""Algorithmic HBM bytes per cell-cycle of the Lagrange + ADI-remap step.

Fixed model (never tuned to measurements): each persistent field crosses HBM
once per pass in which the algorithm reads or writes it; quantities derivable
on chip (pressure, sound speed, node mass, corner vectors, face geometry, cell
centres) are not counted.  Five dependent passes: Lagrange (L), three
directional sweeps (S_x, S_y, S_z) and the finalisation (F).  FP64 words.

  L   : read cell rho, e, q, V0 (32 B); node v, x0, x_lag(n-1) (72 B);
        write cell U (3K+1 words) and L (8 B); node U_dual (5 words), x_lag, v_half (48 B)
  S_d : read + write cell U (2 x 8(3K+1)); node U_dual (2 x 40 B); read node x_lag, v_half, x0 (72 B)
  F   : read cell U, V0, L; node U_dual; write cell rho, e, q (24 B), node v (24 B)

Single environment: 336 + 680 r bytes per cell-cycle, r = nodes / cells
(Sedov 128^3: 1032 B; Sod 100x5x5: 1325 B).  With K environments the cell part
is 80 + 64(3K+1) bytes, plus 8 B of env_id reads when K > 1, plus 128 B per
mixed cell (partial values of two environments read and written in L and F).
"""


def cell_part(nenv: int = 1) -> float:
    b = 80 + 64 * (3 * nenv + 1)
    if nenv > 1:
        b += 8
    return float(b)


NODE_PART = 680.0


def bytes_per_cell_cycle(ncells: int, nnodes: int, nenv: int = 1, mixed_fraction: float = 0.0) -> float:
    r = nnodes / ncells
    b = cell_part(nenv) + NODE_PART * r
    if nenv > 1:
        b += 2 * 4 * 8 * nenv * mixed_fraction
    return b
