"""Python restatement of the device random numbers (Philox4x32-10, Salmon et
al. SC'11) used by the kernels, so tests can predict device-side draws."""
M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32(c, key):
    x, y, z, w = c
    k0, k1 = key & MASK, (key >> 32) & MASK
    for _ in range(10):
        p0 = M0 * x
        p1 = M1 * z
        hi0, lo0 = (p0 >> 32) & MASK, p0 & MASK
        hi1, lo1 = (p1 >> 32) & MASK, p1 & MASK
        x, y, z, w = hi1 ^ y ^ k0, lo1, hi0 ^ w ^ k1, lo0
        k0 = (k0 + W0) & MASK
        k1 = (k1 + W1) & MASK
    return x, y, z, w


def u01(a, b):
    v = ((a >> 5) << 26) | (b >> 6)
    return (v + 1.0) * (1.0 / 9007199254740992.0)


def uniform4(seed, walker, step, purpose):
    r1 = philox4x32((walker & MASK, step & MASK, purpose & MASK, 0x51ED2701), seed)
    r2 = philox4x32((walker & MASK, step & MASK, purpose & MASK, 0x51ED2702), seed)
    return [u01(r1[0], r1[1]), u01(r1[2], r1[3]), u01(r2[0], r2[1]), u01(r2[2], r2[3])]


def umrigar_uniforms(seed, slot, step):
    """The eight uniforms of one Umrigar93 move (lanes 0-3 of the walker's
    warp, two each from their own counter): u[0] picks the branch, u[1..5]
    place the electron, u[6] is the acceptance uniform."""
    u = []
    for k in range(4):
        c = philox4x32((slot & MASK, step & MASK, 8 + k, 0x0A7E5A21), seed)
        u += [u01(c[0], c[1]), u01(c[2], c[3])]
    return u
