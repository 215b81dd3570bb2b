"""A second, pure-Python restatement of AV1 film grain synthesis (spec
7.18.3), written loop for loop from the specification's process
descriptions, to check the C++ oracle's restatement on small frames.

vaco has no grain synthesis (it parses the parameters only,
src/frame_header.rs:1125-1210) and no golden vector exists for it, so the
two restatements and the CUDA kernels can only be checked against each
other: parity of this part is unpinned.  Test infrastructure only."""
import numpy as np


def _round2(x, n):
    return x if n == 0 else (x + (1 << (n - 1))) >> n


def _clip3(lo, hi, x):
    return lo if x < lo else hi if x > hi else x


class _Rng:
    def __init__(self, seed):
        self.r = seed & 0xFFFF

    def get(self, bits):
        r = self.r
        bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1
        r = (r >> 1) | (bit << 15)
        self.r = r
        return (r >> (16 - bits)) & ((1 << bits) - 1)


def film_grain(planes, bd, sub_x, sub_y, mono, p, gauss):
    """planes: list of 2-D uint16 arrays (luma w x h first); p: a
    FilmGrainParams; gauss: 2048 ints.  Returns the output planes."""
    h, w = planes[0].shape
    np_ = 1 if mono else 3
    if not p.apply_grain:
        return [q.copy() for q in planes[:np_]]
    center = 128 << (bd - 8)
    gmin, gmax = -center, (256 << (bd - 8)) - 1 - center
    shift = 12 - bd + p.grain_scale_shift
    lag = p.ar_coeff_lag
    ar_shift = p.ar_coeff_shift_minus_6 + 6

    # generate grain
    rng = _Rng(p.grain_seed)
    luma = [[0] * 82 for _ in range(73)]
    for y in range(73):
        for x in range(82):
            g = gauss[rng.get(11)] if p.num_y_points > 0 else 0
            luma[y][x] = _round2(g, shift)
    for y in range(3, 73):
        for x in range(3, 79):
            s = pos = 0
            done = False
            for dr in range(-lag, 1):
                for dc in range(-lag, lag + 1):
                    if dr == 0 and dc == 0:
                        done = True
                        break
                    s += luma[y + dr][x + dc] * (p.ar_coeffs_y_plus_128[pos] - 128)
                    pos += 1
                if done:
                    break
            luma[y][x] = _clip3(gmin, gmax, luma[y][x] + _round2(s, ar_shift))
    cw, ch = (44 if sub_x else 82), (38 if sub_y else 73)
    chroma = []
    if not mono:
        on = [p.num_cb_points or p.chroma_scaling_from_luma, p.num_cr_points or p.chroma_scaling_from_luma]
        for k, salt in ((0, 0xB524), (1, 0x49D8)):
            rng = _Rng(p.grain_seed ^ salt)
            t = [[0] * cw for _ in range(ch)]
            for y in range(ch):
                for x in range(cw):
                    t[y][x] = _round2(gauss[rng.get(11)] if on[k] else 0, shift)
            chroma.append(t)
        coefs = [p.ar_coeffs_cb_plus_128, p.ar_coeffs_cr_plus_128]
        for y in range(3, ch):
            for x in range(3, cw - 3):
                sums = [0, 0]
                for k in range(2):
                    pos = 0
                    done = False
                    for dr in range(-lag, 1):
                        for dc in range(-lag, lag + 1):
                            c = coefs[k][pos] - 128
                            if dr == 0 and dc == 0:
                                if p.num_y_points > 0:
                                    ly, lx = ((y - 3) << sub_y) + 3, ((x - 3) << sub_x) + 3
                                    l = sum(luma[ly + i][lx + j] for i in range(sub_y + 1) for j in range(sub_x + 1))
                                    sums[k] += _round2(l, sub_x + sub_y) * c
                                done = True
                                break
                            sums[k] += c * chroma[k][y + dr][x + dc]
                            pos += 1
                        if done:
                            break
                for k in range(2):
                    if on[k]:
                        chroma[k][y][x] = _clip3(gmin, gmax, chroma[k][y][x] + _round2(sums[k], ar_shift))
    templates = [luma] + chroma

    # scaling lookup
    def points(plane):
        if plane == 0 or p.chroma_scaling_from_luma:
            n, v, s = p.num_y_points, p.point_y_value, p.point_y_scaling
        elif plane == 1:
            n, v, s = p.num_cb_points, p.point_cb_value, p.point_cb_scaling
        else:
            n, v, s = p.num_cr_points, p.point_cr_value, p.point_cr_scaling
        return n, list(v[:n]), list(s[:n])

    luts = []
    for plane in range(np_):
        n, v, s = points(plane)
        lut = [0] * 256
        if n:
            for x in range(v[0]):
                lut[x] = s[0]
            for i in range(n - 1):
                dy, dx = s[i + 1] - s[i], v[i + 1] - v[i]
                delta = dy * ((65536 + (dx >> 1)) // dx)
                for x in range(dx):
                    lut[v[i] + x] = s[i] + ((x * delta + 32768) >> 16)
            for x in range(v[n - 1], 256):
                lut[x] = s[n - 1]
        luts.append(lut)

    def scale_lut(plane, index):
        sh = bd - 8
        x = index >> sh
        rem = index - (x << sh)
        if bd == 8 or x == 255:
            return luts[plane][x]
        a, b = luts[plane][x], luts[plane][x + 1]
        return a + _round2((b - a) * rem, sh)

    # noise stripes
    stripes = []
    y = 0
    num = 0
    while y < (h + 1) // 2:
        rng = _Rng(p.grain_seed)
        rng.r ^= ((num * 37 + 178) & 255) << 8
        rng.r ^= (num * 173 + 105) & 255
        st = [dict() for _ in range(np_)]
        x = 0
        while x < (w + 1) // 2:
            rand = rng.get(8)
            ox, oy = rand >> 4, rand & 15
            for plane in range(np_):
                psx, psy = (sub_x, sub_y) if plane else (0, 0)
                pox = 6 + ox if psx else 9 + ox * 2
                poy = 6 + oy if psy else 9 + oy * 2
                for i in range(34 >> psy):
                    for j in range(34 >> psx):
                        g = templates[plane][poy + i][pox + j]
                        if psx == 0:
                            if j < 2 and p.overlap_flag and x > 0:
                                old = st[plane][(i, x * 2 + j)]
                                g = old * 27 + g * 17 if j == 0 else old * 17 + g * 27
                                g = _clip3(gmin, gmax, _round2(g, 5))
                            st[plane][(i, x * 2 + j)] = g
                        else:
                            if j == 0 and p.overlap_flag and x > 0:
                                old = st[plane][(i, x + j)]
                                g = _clip3(gmin, gmax, _round2(old * 23 + g * 22, 5))
                            st[plane][(i, x + j)] = g
            x += 16
        stripes.append(st)
        num += 1
        y += 16

    def noise(plane, y, x):
        psy = sub_y if plane else 0
        n = y >> (5 - psy)
        i = y - (n << (5 - psy))
        g = stripes[n][plane][(i, x)]
        if psy == 0:
            if i < 2 and n > 0 and p.overlap_flag:
                old = stripes[n - 1][plane][(i + 32, x)]
                g = old * 27 + g * 17 if i == 0 else old * 17 + g * 27
                g = _clip3(gmin, gmax, _round2(g, 5))
        elif i < 1 and n > 0 and p.overlap_flag:
            old = stripes[n - 1][plane][(i + 16, x)]
            g = _clip3(gmin, gmax, _round2(old * 23 + g * 22, 5))
        return g

    if p.clip_to_restricted_range:
        lo, hi_l = 16 << (bd - 8), 235 << (bd - 8)
        hi_c = hi_l if p.mc_identity else 240 << (bd - 8)
    else:
        lo, hi_l = 0, (256 << (bd - 8)) - 1
        hi_c = hi_l
    sshift = p.grain_scaling_minus_8 + 8
    maxv = (1 << bd) - 1
    out = [q.copy() for q in planes[:np_]]
    src = [q.astype(np.int64) for q in planes[:np_]]
    if p.num_y_points > 0:
        for y in range(h):
            for x in range(w):
                o = int(src[0][y, x])
                out[0][y, x] = _clip3(lo, hi_l, o + _round2(scale_lut(0, o) * noise(0, y, x), sshift))
    for plane in range(1, np_):
        n_points = p.num_cb_points if plane == 1 else p.num_cr_points
        if not (n_points > 0 or p.chroma_scaling_from_luma):
            continue
        mult = p.cb_mult if plane == 1 else p.cr_mult
        lmult = p.cb_luma_mult if plane == 1 else p.cr_luma_mult
        offset = p.cb_offset if plane == 1 else p.cr_offset
        ph, pw = (h + sub_y) >> sub_y, (w + sub_x) >> sub_x
        for y in range(ph):
            for x in range(pw):
                ly, lx = y << sub_y, x << sub_x
                lnx = min(lx + 1, w - 1)
                avg = _round2(int(src[0][ly, lx]) + int(src[0][ly, lnx]), 1) if sub_x else int(src[0][ly, lx])
                o = int(src[plane][y, x])
                if p.chroma_scaling_from_luma:
                    merged = avg
                else:
                    comb = avg * (lmult - 128) + o * (mult - 128)
                    merged = _clip3(0, maxv, (comb >> 6) + ((offset - 256) << (bd - 8)))
                out[plane][y, x] = _clip3(lo, hi_c, o + _round2(scale_lut(plane, merged) * noise(plane, y, x), sshift))
    return out
