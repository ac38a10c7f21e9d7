"""The tuning database: TTC's SQLite schema (ttc.py:205-367, sql_util.py:8-121 in the TTC project)
with one added column, `variant.tuning`, holding the B200 schedule (JSON of ttcb_tuning fields).

Tables `size`, `permutation`, `measurements`, `loopOrder`, `variant` and the views `joined` and
`fastest0Percent` keep TTC's names and columns, so TTC's plotting and queries read it unchanged. A
measurement is keyed like TTC's lookup (sql_util.py:55-77): sizes, permutation, floatTypeA/B,
beta == 0 or not, numThreads >= requested, hotA, hotB and the architecture (device name). Queries
use bound parameters. A corrupt or locked database is reported as `DatabaseUnavailable` so callers
fall back to a measured search.
"""
from __future__ import annotations

import json
import sqlite3
from typing import Optional

MAXDIM = 10


class DatabaseUnavailable(RuntimeError):
    pass


SCHEMA = [
    """CREATE TABLE IF NOT EXISTS 'size' ('size_id' INTEGER NOT NULL PRIMARY KEY AUTOINCREMENT,
       'size0' INTEGER NULL, 'size1' INTEGER NULL, 'size2' INTEGER NULL, 'size3' INTEGER NULL,
       'size4' INTEGER NULL, 'size5' INTEGER NULL, 'size6' INTEGER NULL, 'size7' INTEGER NULL,
       'size8' INTEGER NULL, 'size9' INTEGER NULL)""",
    """CREATE TABLE IF NOT EXISTS 'permutation' ('permutation_id' INTEGER NOT NULL PRIMARY KEY AUTOINCREMENT,
       'idx0' INTEGER NULL, 'idx1' INTEGER NULL, 'idx2' INTEGER NULL, 'idx3' INTEGER NULL, 'idx4' INTEGER NULL,
       'idx5' INTEGER NULL, 'idx6' INTEGER NULL, 'idx7' INTEGER NULL, 'idx8' INTEGER NULL, 'idx9' INTEGER NULL)""",
    """CREATE TABLE IF NOT EXISTS 'measurements' ('measurement_id' INTEGER NOT NULL PRIMARY KEY AUTOINCREMENT,
       'dim' INTEGER NULL, 'host' VARCHAR(45) NULL, 'architecture' VARCHAR(45) NULL, 'version' VARCHAR(45) NULL,
       'alpha' FLOAT NULL, 'beta' FLOAT NULL, 'numThreads' INTEGER NULL, 'compiler_version' VARCHAR(60) NULL,
       'floatTypeA' VARCHAR(45) NULL, 'floatTypeB' VARCHAR(45) NULL, 'top1' FLOAT NULL, 'top5' FLOAT NULL,
       'compilationTime' FLOAT NULL, 'measuringTime' FLOAT NULL, 'referenceBandwidth' FLOAT NULL,
       'size_id' INTEGER NULL, 'permutation_id' INTEGER NULL, 'hotA' INTEGER NULL, 'hotB' INTEGER NULL,
       FOREIGN KEY ('size_id') REFERENCES 'size' ('size_id'),
       FOREIGN KEY ('permutation_id') REFERENCES 'permutation' ('permutation_id'))""",
    """CREATE TABLE IF NOT EXISTS 'loopOrder' ('loopOrder_id' INTEGER NOT NULL PRIMARY KEY AUTOINCREMENT,
       'idx0' INTEGER NULL, 'idx1' INTEGER NULL, 'idx2' INTEGER NULL, 'idx3' INTEGER NULL, 'idx4' INTEGER NULL,
       'idx5' INTEGER NULL, 'idx6' INTEGER NULL, 'idx7' INTEGER NULL, 'idx8' INTEGER NULL, 'idx9' INTEGER NULL)""",
    """CREATE TABLE IF NOT EXISTS 'variant' ('variant_id' INTEGER NOT NULL PRIMARY KEY AUTOINCREMENT,
       'blockA' INTEGER NULL, 'blockB' INTEGER NULL, 'prefetchDistance' INTEGER NULL, 'bandwidth' FLOAT NULL,
       'time' FLOAT NULL, 'tlbMisses' FLOAT NULL, 'l2misses' FLOAT NULL, 'rankLoopOrder' INTEGER NULL,
       'rankBlocking' INTEGER NULL, 'measurement_id' INTEGER NULL, 'loopOrder_id' INTEGER NULL,
       'tuning' TEXT NULL,
       FOREIGN KEY ('measurement_id') REFERENCES 'measurements' ('measurement_id'),
       FOREIGN KEY ('loopOrder_id') REFERENCES 'loopOrder' ('loopOrder_id'))""",
    """CREATE VIEW IF NOT EXISTS 'joined' AS SELECT * FROM measurements JOIN size ON measurements.size_id =
       size.size_id JOIN permutation ON measurements.permutation_id = permutation.permutation_id JOIN variant
       ON variant.measurement_id = measurements.measurement_id""",
    """CREATE VIEW IF NOT EXISTS 'fastest0Percent' AS SELECT * FROM measurements JOIN (
       SELECT v2.* FROM (SELECT *, max(bandwidth) AS maxBandwidth FROM variant GROUP BY measurement_id) v1
       INNER JOIN variant v2 ON v1.measurement_id = v2.measurement_id WHERE v2.bandwidth >= (1.0 * v1.maxBandwidth)
       ) fast ON measurements.measurement_id = fast.measurement_id""",
]


def connect(path: str) -> sqlite3.Connection:
    try:
        con = sqlite3.connect(path, timeout=2.0)
        cur = con.cursor()
        for cmd in SCHEMA:
            cur.execute(cmd)
        con.commit()
        return con
    except sqlite3.Error as e:
        raise DatabaseUnavailable(f"tuning database {path}: {e}") from e


def _row_where(prefix: str, values) -> tuple[str, list]:
    parts, args = [], []
    for i in range(MAXDIM):
        if i < len(values):
            parts.append(f"{prefix}{i} = ?")
            args.append(int(values[i]))
        else:
            parts.append(f"{prefix}{i} IS NULL")
    return " AND ".join(parts), args


def _get_or_insert(cur, table: str, key: str, prefix: str, values) -> int:
    where, args = _row_where(prefix, values)
    cur.execute(f"SELECT {key} FROM {table} WHERE {where}", args)
    row = cur.fetchone()
    if row:
        return int(row[0])
    cols = ", ".join(f"{prefix}{i}" for i in range(len(values)))
    marks = ", ".join("?" for _ in values)
    cur.execute(f"INSERT INTO {table} ({cols}) VALUES ({marks})", [int(v) for v in values])
    return int(cur.lastrowid)


def getSizeId(cur, size) -> int:
    where, args = _row_where("size", size)
    cur.execute(f"SELECT size_id FROM size WHERE {where}", args)
    row = cur.fetchone()
    return int(row[0]) if row else -1


def getPermId(cur, perm) -> int:
    where, args = _row_where("idx", perm)
    cur.execute(f"SELECT permutation_id FROM permutation WHERE {where}", args)
    row = cur.fetchone()
    return int(row[0]) if row else -1


def getMeasurementId(cur, sizeId, permId, floatTypeA, floatTypeB, beta, numThreads, hotA, hotB, architecture) -> int:
    beta_clause = "beta != 0" if beta != 0 else "beta = 0"
    cur.execute(f"""SELECT measurement_id FROM measurements WHERE size_id = ? AND permutation_id = ? AND
                    floatTypeA = ? AND floatTypeB = ? AND {beta_clause} AND numThreads >= ? AND hotA = ? AND
                    hotB = ? AND architecture = ? ORDER BY measurement_id DESC""",
                (sizeId, permId, floatTypeA, floatTypeB, numThreads, hotA, hotB, architecture))
    row = cur.fetchone()
    return int(row[0]) if row else -1


def getBestImplementation(cur, measurementId):
    """(blockA, blockB, loopOrder_id, prefetchDistance, bandwidth, tuning dict) of the fastest variant."""
    cur.execute("""SELECT blockA, blockB, loopOrder_id, prefetchDistance, bandwidth, tuning FROM variant
                   WHERE measurement_id = ? ORDER BY bandwidth DESC""", (measurementId,))
    row = cur.fetchone()
    if not row:
        return -1
    tuning = json.loads(row[5]) if row[5] else {}
    return (row[0], row[1], row[2], row[3], row[4], tuning)


def lookup(path: str, size, perm, floatTypeA, floatTypeB, beta, architecture) -> Optional[dict]:
    """The stored best schedule for a (fused) problem, or None. Raises DatabaseUnavailable."""
    con = connect(path)
    try:
        cur = con.cursor()
        sid = getSizeId(cur, size)
        pid = getPermId(cur, perm)
        if sid < 0 or pid < 0:
            return None
        mid = getMeasurementId(cur, sid, pid, floatTypeA, floatTypeB, beta, 0, 0, 0, architecture)
        if mid < 0:
            return None
        best = getBestImplementation(cur, mid)
        if best == -1:
            return None
        return {"tuning": best[5], "bandwidth": best[4]}
    except sqlite3.Error as e:
        raise DatabaseUnavailable(str(e)) from e
    finally:
        con.close()


def insert(path: str, size, perm, floatTypeA, floatTypeB, alpha, beta, architecture, host, variants,
           measuring_time: float, reference_bw: float = -1.0) -> int:
    """Stores one tuning run. `variants`: dicts with tuning, bandwidth (GiB/s), time (s), rank."""
    con = connect(path)
    try:
        cur = con.cursor()
        sid = _get_or_insert(cur, "size", "size_id", "size", size)
        pid = _get_or_insert(cur, "permutation", "permutation_id", "idx", perm)
        cur.execute("""INSERT INTO measurements (dim, host, architecture, version, alpha, beta, numThreads,
                       compiler_version, floatTypeA, floatTypeB, top1, top5, compilationTime, measuringTime,
                       referenceBandwidth, size_id, permutation_id, hotA, hotB)
                       VALUES (?, ?, ?, ?, ?, ?, 0, ?, ?, ?, 0, 0, 0, ?, ?, ?, ?, 0, 0)""",
                    (len(perm), host, architecture, "ttc_b200", float(complex(alpha).real),
                     float(complex(beta).real) if complex(beta) != 0 else 0.0, "nvcc sm_100a", floatTypeA,
                     floatTypeB, measuring_time, reference_bw, sid, pid))
        mid = int(cur.lastrowid)
        for v in variants:
            t = v["tuning"]
            loop = list(t["raster"]) if t.get("raster") else [t.get("loop_order", 0)]
            lid = _get_or_insert(cur, "loopOrder", "loopOrder_id", "idx", loop)
            cur.execute("""INSERT INTO variant (blockA, blockB, prefetchDistance, bandwidth, time, tlbMisses,
                           l2misses, rankLoopOrder, rankBlocking, measurement_id, loopOrder_id, tuning)
                           VALUES (?, ?, 0, ?, ?, -1, 0, ?, ?, ?, ?, ?)""",
                        (int(v.get("blockA", 0)), int(v.get("blockB", 0)), float(v["bandwidth"]), float(v["time"]),
                         int(v.get("rank", 0)), int(v.get("rank", 0)), mid, lid, json.dumps(t, sort_keys=True)))
        con.commit()
        return mid
    except sqlite3.Error as e:
        raise DatabaseUnavailable(str(e)) from e
    finally:
        con.close()
