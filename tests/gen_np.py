"""Numpy restatement of the seeded synthetic lineitem generator (test infrastructure).

The product generates rows in C++/CUDA (tpchq01_gpu_b200/csrc/q1_common.cuh, gen_row); this
independent numpy version produces the same rows and is used to feed the oracle and to check
the product's host and device generators bit for bit.

Distribution (the lineitem columns Q1 reads):
  orderdate  uniform day in [1992-01-01, 1998-08-02]; shipdate = orderdate + U{1..121};
  receiptdate = shipdate + U{1..30}; quantity U{1..50}; unit price U[90000, 209899] cents;
  extendedprice = quantity * unit price; discount U{0..10}; tax U{0..8} (hundredths);
  returnflag R/A (1/2 each) if receiptdate <= 1995-06-17 else N;
  linestatus O if shipdate > 1995-06-17 else F.
"""
import numpy as np

M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)
GOLDEN = np.uint64(0x9E3779B97F4A7C15)
SEED_XOR = np.uint64(0x5DEECE66DA3B9F21)

ORDER_FIRST = 727563  # 1992-01-01
ORDER_LAST = 729968   # 1998-08-02
CURRENT = 728826      # 1995-06-17
FRAME = 727563

F_ORDER, F_SHIP, F_RECEIPT, F_QTY, F_PRICE, F_DISC, F_TAX, F_RF, F_KEY = range(9)


def mix64(z):
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
    return z ^ (z >> np.uint64(31))


def gen_key(seed):
    return mix64(np.uint64(seed) ^ SEED_XOR)


def gen_bits(key, rows, field):
    with np.errstate(over="ignore"):
        x = key + (rows * np.uint64(16) + np.uint64(field)) * GOLDEN
    return (mix64(x) >> np.uint64(32)).astype(np.uint64)


def uniform(bits, span):
    return ((bits * np.uint64(span)) >> np.uint64(32)).astype(np.int64)


def generate(seed, first_row, rows):
    """Reference-typed columns (cpu/tpch_kit.hpp lineitem): int32 shipdate day numbers,
    int64 hundredths for discount/tax/quantity, int64 cents for extendedprice, chars for flags."""
    key = gen_key(seed)
    r = np.arange(first_row, first_row + rows, dtype=np.uint64)
    order = ORDER_FIRST + uniform(gen_bits(key, r, F_ORDER), ORDER_LAST - ORDER_FIRST + 1)
    ship = order + 1 + uniform(gen_bits(key, r, F_SHIP), 121)
    receipt = ship + 1 + uniform(gen_bits(key, r, F_RECEIPT), 30)
    qty = 1 + uniform(gen_bits(key, r, F_QTY), 50)
    unit = 90000 + uniform(gen_bits(key, r, F_PRICE), 209899 - 90000 + 1)
    disc = uniform(gen_bits(key, r, F_DISC), 11)
    tax = uniform(gen_bits(key, r, F_TAX), 9)
    coin = (gen_bits(key, r, F_RF) >> np.uint64(31)).astype(bool)
    rf = np.where(receipt <= CURRENT, np.where(coin, ord("R"), ord("A")), ord("N")).astype(np.uint8)
    ls = np.where(ship > CURRENT, ord("O"), ord("F")).astype(np.uint8)
    return {
        "shipdate": ship.astype(np.int32),
        "discount": disc.astype(np.int64),
        "extendedprice": (qty * unit).astype(np.int64),
        "tax": tax.astype(np.int64),
        "quantity": (qty * 100).astype(np.int64),
        "returnflag": rf.view("S1"),
        "linestatus": ls.view("S1"),
    }


def group_keys_uniform(seed, first_row, rows, num_groups):
    key = gen_key(seed)
    r = np.arange(first_row, first_row + rows, dtype=np.uint64)
    return uniform(gen_bits(key, r, F_KEY), num_groups).astype(np.uint32)


def zipf_cdf(num_groups, s=1.1):
    """uint32 inverse-CDF thresholds of Zipf(s) over ranks 1..G (key = rank - 1)."""
    w = 1.0 / np.power(np.arange(1, num_groups + 1, dtype=np.float64), s)
    c = np.cumsum(w) / w.sum()
    t = np.minimum(np.floor(c * 4294967296.0), 4294967295.0).astype(np.uint64)
    t[-1] = 0xFFFFFFFF
    return t.astype(np.uint32)


def group_keys_cdf(seed, first_row, rows, cdf):
    key = gen_key(seed)
    r = np.arange(first_row, first_row + rows, dtype=np.uint64)
    b = gen_bits(key, r, F_KEY).astype(np.uint32)
    return np.searchsorted(cdf, b, side="left").astype(np.uint32)


def compress(cols, packing="pair"):
    """Compressed layout (src/main.cu:773-803): uint16 day offset, uint8 disc/tax, uint32 cents,
    uint8 whole-unit quantity, flags bit-packed LSB first (src/bit_operations.hpp)."""
    n = len(cols["shipdate"])
    out = {
        "shipdate": (cols["shipdate"] - FRAME).astype(np.uint16),
        "discount": cols["discount"].astype(np.uint8),
        "extendedprice": cols["extendedprice"].astype(np.uint32),
        "tax": cols["tax"].astype(np.uint8),
        "quantity": (cols["quantity"] // 100).astype(np.uint8),
    }
    rfc = cols["returnflag"].view(np.uint8)
    lsc = cols["linestatus"].view(np.uint8)
    rf = np.where(rfc == ord("R"), 2, 0) + np.where(rfc == ord("N"), 1, 0)
    ls = np.where(lsc == ord("F"), 0, 1)
    group = (rf << 1) + ls
    if packing == "pair":
        present = sorted(set(np.unique(group).tolist()))
        assert len(present) <= 4
        code_of = {g: i for i, g in enumerate(present)}
        lut = np.zeros(6, dtype=np.int64)
        for g, c in code_of.items():
            lut[g] = c
        codes = lut[group]
        out["flags"] = pack_bits(codes, 2, n)
        out["pair_group"] = np.array(present + [0] * (4 - len(present)), dtype=np.uint8)
        out["num_pair_codes"] = len(present)
    else:
        out["returnflag"] = pack_bits(rf, 2, n)
        out["linestatus"] = pack_bits(ls, 1, n)
    return out


def pack_bits(values, bits, n):
    per = 32 // bits
    words = (n + per - 1) // per
    v = np.zeros(words * per, dtype=np.uint64)
    v[:n] = values
    v = v.reshape(words, per)
    shifts = (np.arange(per, dtype=np.uint64) * np.uint64(bits))
    return np.bitwise_or.reduce(v << shifts, axis=1).astype(np.uint32)


def filter_bitmap(c_shipdate, cutoff_day):
    n = len(c_shipdate)
    bits = (c_shipdate.astype(np.int64) <= cutoff_day - FRAME).astype(np.uint64)
    return pack_bits(bits, 1, n)
