"""Test infrastructure: a second, independent restatement of the reference's skyrmion counting
stage in plain Python/numpy, written from the Fortran text, used to cross-check the C oracle
(ora_skyrmion_number) and the device on textures with a known winding number.  Never called by
the product.

Follows src/reciprocalSpaceProcesses.f90 (rsp):
- Gaussian_filter_2d (rsp:814-858): 5 x 5 kernel exp(-(l^2 + m^2) / (2 sigma^2)) normalised,
  applied as buffer(i, j) = sum_{l,m=1..5} array(i - l, j - m) G(l, m), periodic, which shifts
  the density by (3, 3);
- calculate_skyrmion_number (rsp:627-812) after its interpolation step: mask |d| > q max|d|;
  a cell starts a region when it is masked, unvisited and a local maximum of |d| against its 8
  neighbours taken modulo the COARSE cell counts (rsp:711-712); the region grows by a stack
  flood fill over masked, unvisited, downhill neighbours (add_neighbors_to_stack, rsp:582-625:
  a neighbour index below 1 becomes the COARSE count and one above the coarse count becomes 1,
  rsp:596-607; downhill = |d(i,j)| >= |d(n)| - 1e-10); the final loop runs over
  CELLS and adds nint(sign(acc)) for every cell of an unmerged region whose |acc| is within 0.05
  of particle_number (rsp:764-773), and marks pairs of neighbouring regions (coarse modulo
  again) merged when their sum is.
"""
from __future__ import annotations

import numpy as np


def gaussian_filter_2d(a, sigma):
    k = 2
    G = np.zeros((2 * k + 1, 2 * k + 1))
    for i in range(1, 2 * k + 2):
        for j in range(1, 2 * k + 2):
            G[i - 1, j - 1] = np.exp(-((i - k - 1) ** 2 + (j - k - 1) ** 2) / (2 * sigma ** 2))
    G /= G.sum()
    out = np.zeros_like(a)
    for l in range(1, 2 * k + 2):
        for m in range(1, 2 * k + 2):
            out += G[l - 1, m - 1] * np.roll(np.roll(a, l, 0), m, 1)   # array(i - l, j - m)
    return out


def skyrmion_number(dens, ncx, ncy, q_threshold, particle_number, sigma):
    """The count of calculate_skyrmion_number on the (fx, fy) fine density with coarse cell
    counts (ncx, ncy); returns (count, region sums)."""
    d = gaussian_filter_2d(np.array(dens, dtype=np.float64), sigma)
    n, l = d.shape
    ad = np.abs(d)
    mask = ad > q_threshold * ad.max()
    visited = np.zeros((n, l), bool)
    region = np.zeros((n, l), int)
    accs = []
    for i in range(n):
        for j in range(l):
            local_max = True
            for di in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    if di == 0 and dj == 0:
                        continue
                    if ad[i, j] < ad[(i + di) % ncx, (j + dj) % ncy]:
                        local_max = False
            if not (mask[i, j] and not visited[i, j] and local_max):
                continue
            visited[i, j] = True
            accs.append(d[i, j])
            region[i, j] = len(accs)
            stack, in_stack = [], np.zeros((n, l), bool)

            def push(ci, cj):
                for di in (-1, 0, 1):
                    for dj in (-1, 0, 1):
                        x, y = ci + di, cj + dj            # 0-based form of the coarse wrap
                        x = ncx - 1 if x < 0 else (0 if x > ncx - 1 else x)
                        y = ncy - 1 if y < 0 else (0 if y > ncy - 1 else y)
                        if in_stack[x, y]:
                            continue
                        if not visited[x, y] and mask[x, y] and ad[ci, cj] >= ad[x, y] - 1e-10:
                            stack.append((x, y))
                            in_stack[x, y] = True

            push(i, j)
            while stack:
                x, y = stack.pop()
                if not visited[x, y]:
                    accs[-1] += d[x, y]
                    visited[x, y] = True
                    push(x, y)
                    region[x, y] = len(accs)
    merged = [False] * len(accs)
    count = 0
    for i in range(n):
        for j in range(l):
            r1 = region[i, j] - 1
            if r1 < 0 or merged[r1]:
                continue
            if abs(abs(accs[r1]) - particle_number) < 0.05:
                count += int(np.sign(accs[r1]))
                continue
            for di in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    if di == 0 and dj == 0:
                        continue
                    r2 = region[(i + di) % ncx, (j + dj) % ncy] - 1
                    if r2 < 0 or merged[r2]:
                        continue
                    if abs(abs(accs[r1] + accs[r2]) - particle_number) < 0.05:
                        merged[r1] = merged[r2] = True
    return count, accs
