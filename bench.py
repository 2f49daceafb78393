"""Batched chunk decode benchmark: decoded GB/s per B200 at q=6.

Workload (per rank): 64 synthetic 256^3 u8 chunks (1 GiB raw; seeds
rank*64 .. rank*64+63, air fraction 30-60 %), encoded at q=6 into an archive
whose bytes are resident in HBM; one step decodes every block of every chunk
through a graph-captured decode plan (entropy stage + reconstruction stage).

  value     decoded bytes of all ranks / max-over-ranks step time (CUDA events
            on the launching stream; the L2 is flushed by a 256 MiB write
            between steps, outside the timed events)
  e2e       the same metric through mc_b200_decode_chunk_blobs with HOST
            buffers: compressed blobs host->device and voxels device->host
            inside every step (pinned host memory)
  roofline  the dominant kernel (entropy stage) timed alone with CUDA events,
            decoded bytes per launch / its time, against the measured HBM peak
  cpu_baseline  the reference's own decode (its sources built with its default
            optimisation flags, oracle/_ref/libmcref_fast.so) on this host's
            cores, mc_archive_decode_chunk(nthreads=0), rank 0 at N=1 only

`--impl reference` runs only the reference's CPU decode of the same workload
(rank 0; other ranks exit) and prints the same JSON line with "impl": "reference".
Multi-GPU: python -m torch.distributed.run --nproc-per-node N bench.py --gpus N
(weak scaling: every rank decodes its own 64 chunks; no data-path collective).
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "matter-compressor_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from shard import Dist, chunk_seeds, air_fraction  # noqa: E402

CHUNK = 256 ** 3
METRIC = "decoded GB/s per B200 at q=6 (bit-exact); p50/p99 block-request latency"
HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) per decoded chunk of the entropy stage, measured
# with ncu on a 16-chunk case and scaled per chunk
# (profiles/k_entropy_decode_q6_16chunks.md).
ENTROPY_DRAM_BYTES_PER_CHUNK = (12.763136e6 + 3.737856e6) / 16


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--chunks", type=int, default=64)
    p.add_argument("--q", type=float, default=6.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--q-sweep", action="store_true",
                   help="decode: one JSON line per quality in 1, 3, 6, 12 (each with its autotuned launch shape "
                        "and the reference's CPU decode of the same archive)")
    p.add_argument("--workload", default="decode", choices=["decode", "serve", "regions", "encode", "deblock", "pyramid"],
                   help="decode: batched chunk decode (the headline line); serve: request-serving sweep; "
                        "regions: dataloader region batch; encode: preset-ladder batched encode; "
                        "deblock: decode-side deblocking of the decoded chunks; pyramid: LOD pyramid build")
    p.add_argument("--rates", default="1000,10000,30000,100000,300000,1000000",
                   help="serve: offered request rates (req/s)")
    p.add_argument("--serve-seconds", type=float, default=0.3, help="serve: arrival window per rate")
    return p.parse_args()


def make_volumes(seeds, device):
    import volumes
    out = torch.empty((len(seeds), 256, 256, 256), dtype=torch.uint8, device=device)
    for i, s in enumerate(seeds):
        out[i] = volumes.region(s, (0, 0, 256 * i), (256, 256, 256), air_fraction(i), device=device)
    return out


class Clocks:
    """nvidia-smi sampling of the GPU's SM clock and throttle reasons while running."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc, self.path = None, None

    def start(self):
        try:
            uuid = str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
            ident = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            ident = "0"
        self.path = tempfile.mktemp(suffix=".csv")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", ident, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms",
                 "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                rows.append(parts)
        os.remove(self.path)
        if not rows:
            return None

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [num(r[0]) for r in rows if num(r[0]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[4:8]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(rows[0][1]),
                "reasons": reasons, "samples": len(rows)}


def hbm_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def blobs_of(path, offs):
    """Chunk blobs of an archive file (header, fmap, bitmap, lengths, payloads)."""
    data = np.fromfile(path, np.uint8)
    out = []
    for co in offs:
        fml = int(data[co + 12]) | (int(data[co + 13]) << 8)
        bm = data[co + 14 + fml:co + 14 + fml + 512]
        npres = int(np.unpackbits(bm).sum())
        lens = data[co + 14 + fml + 512:co + 14 + fml + 512 + 2 * npres].view(np.uint16).astype(np.int64)
        n = 14 + fml + 512 + 2 * npres + int(lens.sum())
        out.append(data[co:co + n])
    return out


# ------------------------------------------------------------------ reference CPU decode
def reference_decode(path, nchunks, q, steps, warmup, min_seconds=0.0):
    """The reference's own mc_archive_decode_chunk(nthreads=0) over the archive."""
    from mcb200 import McLib
    from oracle import REF_FAST_LIB
    ref = McLib(REF_FAST_LIB, b200=False)
    ref.L.mc_codec_init()
    a = ref.open(path, 256 * nchunks, 256, 256, q)
    offs = [a.chunk_offset(0, 0, 0, c) for c in range(nchunks)]
    out = np.empty(CHUNK, np.uint8)
    for _ in range(warmup):
        a.decode_chunk(offs[0], out, 0)
    times, done = [], 0
    t_start = time.perf_counter()
    for _ in range(max(steps, 1)):
        t0 = time.perf_counter()
        for co in offs:
            a.decode_chunk(co, out, 0)
        times.append(time.perf_counter() - t0)
        done += 1
        if min_seconds and time.perf_counter() - t_start > min_seconds:
            break
    a.close()
    cores = min(os.cpu_count() or 4, 16)   # the reference's thread cap (src/mc_archive.c:805-809)
    gbs = nchunks * CHUNK / statistics.mean(times) / 1e9
    return gbs, cores, done, times


def host_read_regions_ms(a, boxes, dz, dy, dx, stride, reps=3):
    """Median ms of mc_archive_read_regions (host output) over reps calls after
    one warm-up call, into one output buffer whose pages are touched first: the
    steady cost of the call, without first-call allocations or the page faults
    of fresh output memory. Returns (ms, output)."""
    import ctypes as C
    from mcb200 import McBox
    n = len(boxes)
    arr = (McBox * n)(*[McBox(*b) for b in boxes])
    out = np.empty(stride * (n - 1) + dz * dy * dx, np.uint8)
    out.fill(0)
    ts = []
    for r in range(reps + 1):
        t0 = time.perf_counter()
        a.L.mc_archive_read_regions(a.a, 0, C.cast(arr, C.c_void_p), n, dz, dy, dx, out.ctypes.data, stride, 0)
        if r:
            ts.append((time.perf_counter() - t0) * 1e3)
    return statistics.median(ts), out


def block_latency(a, offs, picks, skip=20):
    """ms per mc_archive_decode_block call on (chunk, block) picks; the first
    `skip` calls warm up."""
    out = np.empty(4096, np.uint8)
    dst = C.c_void_p(out.ctypes.data)
    lat = []
    for c, bi in picks:
        t0 = time.perf_counter()
        a.L.mc_archive_decode_block(a.a, offs[c], bi >> 8, (bi >> 4) & 15, bi & 15, dst)
        lat.append((time.perf_counter() - t0) * 1e3)
    return lat[skip:]


def plain_chunk_blocks_ms(a, co):
    """ms for 4096 mc_archive_decode_block calls covering one chunk."""
    out = np.empty(4096, np.uint8)
    dst = C.c_void_p(out.ctypes.data)
    for bi in range(64):   # warm
        a.L.mc_archive_decode_block(a.a, co, bi >> 8, (bi >> 4) & 15, bi & 15, dst)
    t0 = time.perf_counter()
    for bi in range(4096):
        a.L.mc_archive_decode_block(a.a, co, bi >> 8, (bi >> 4) & 15, bi & 15, dst)
    return (time.perf_counter() - t0) * 1e3


def reference_block_latency(path, nchunks, q, picks):
    """The reference's own decode_block on the same blocks, and its plain
    4096-call pass over chunk 0 (one host thread, default-flag build)."""
    from mcb200 import McLib
    from oracle import REF_FAST_LIB
    ref = McLib(REF_FAST_LIB, b200=False)
    ref.L.mc_codec_init()
    with ref.open(path, 256 * nchunks, 256, 256, q) as r:
        offs = [r.chunk_offset(0, 0, 0, c) for c in range(nchunks)]
        lat = block_latency(r, offs, picks)
        plain = plain_chunk_blocks_ms(r, offs[0])
    return lat, plain


def build_reference_archive(path, vox_host, q):
    from mcb200 import McLib
    from oracle import REF_FAST_LIB
    ref = McLib(REF_FAST_LIB, b200=False)
    ref.L.mc_codec_init()
    n = len(vox_host)
    with ref.open(path, 256 * n, 256, 256, q) as a:
        for c in range(n):
            assert a.append_par(0, 0, 0, c, vox_host[c], q, 0) == 0


def config(args, world):
    return {"workload": f"batched chunk decode: {args.chunks} x 256^3 u8 chunks per GPU "
                        f"({args.chunks * CHUNK / 2**30:.2f} GiB), q={args.q:g}, archive resident in HBM, "
                        "one graph-captured decode plan per step",
            "chunks_per_gpu": args.chunks, "q": args.q, "air_fraction": "30-60%",
            "generator": "4-octave value noise (period 32) 40..220 + N(0,6^2), 2-octave air mask",
            "l2": "flushed by a 256 MiB write between timed steps",
            "parallelism": f"{world} x independent chunk shards"}



# ------------------------------------------------------------------ other configurations
VOLUME_DIMS = (1024, 2048, 2048)   # z, y, x voxels of the dataloader / serving volume


def pct(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q))


def run_serve(args):
    """Serving sweep: Poisson mixes of block / region / chunk reads at each
    offered rate through the serving loop (device outputs, 8 GiB cache), and
    the same kinds of requests one at a time through the plain per-call API."""
    import workloads
    from mcb200 import McLib, Server
    lib = McLib.product()
    td = tempfile.mkdtemp()
    path = os.path.join(td, "serve.mca")
    t0 = time.perf_counter()
    a, nch = workloads.build_volume_archive(lib, path, VOLUME_DIMS, lods=4, q=args.q)
    build_s = time.perf_counter() - t0
    outs = [torch.empty(n, dtype=torch.uint8, device="cuda") for n in (4096, 128 ** 3, 256 ** 3)]
    rates = [float(r) for r in args.rates.split(",")]

    def trace_requests(tr):
        reqs = []
        for i in range(len(tr)):
            k = int(tr.kind[i])
            z, y, x, dz, dy, dx = (int(v) for v in tr.req[i, :6])
            reqs.append(Server.request(workloads.Trace.KINDS[k], int(tr.lod[i]), z, y, x, outs[k].data_ptr(),
                                       dz, dy, dx))
        return reqs

    rows = []
    # one server for the whole sweep (steady state): a warm-up trace fills the
    # cache and grows every buffer before the measured rates
    with Server(a, 8 << 30, 512 << 20) as srv:
        wt = workloads.Trace(7, 20000, 30000.0, VOLUME_DIMS, lods=4)
        rc, _ = srv.replay(trace_requests(wt), wt.arrival_ns)
        assert rc == 0, "serving warm-up failed"
        for ri, rate in enumerate(rates):
            n = max(200, min(200000, int(rate * args.serve_seconds)))
            tr = workloads.Trace(1000 + ri, n, rate, VOLUME_DIMS, lods=4)
            s0 = srv.stats()
            rc, lat = srv.replay(trace_requests(tr), tr.arrival_ns)
            st = {k: v - s0[k] for k, v in srv.stats().items()}
            assert rc == 0, "serving replay failed"
            end = float((tr.arrival_ns.astype(np.float64) + lat.astype(np.float64)).max()) / 1e9
            nbytes = sum(tr.out_bytes(i) for i in range(n))
            lat_ms = lat.astype(np.float64) / 1e6
            rows.append({"offered_req_s": rate, "requests": n, "achieved_req_s": round(n / end, 1),
                         "gbs": round(nbytes / end / 1e9, 3), "p50_ms": round(pct(lat_ms, 50), 4),
                         "p99_ms": round(pct(lat_ms, 99), 4),
                         "p99_ms_by_kind": {workloads.Trace.NAMES[k]: round(pct(lat_ms[tr.kind == k], 99), 4)
                                            for k in range(3) if (tr.kind == k).any()},
                         "hit_rate": round(st["hits"] / max(1, st["hits"] + st["misses"]), 4),
                         "batches": st["batches"]})
    # plain per-call drop-in on the same mix, one call at a time: with device
    # outputs (like for like with the server's device outputs) and with host
    # outputs (the reference's own call signatures)
    tr = workloads.Trace(99, 400, 1e4, VOLUME_DIMS, lods=4)
    plain_dev = plain_per_call(a, tr, outs, device=True)
    plain_host = plain_per_call(a, tr, None, device=False)
    # the plain per-call path under the same open-loop arrivals as the server:
    # one caller thread issues each request at its arrival time (or as soon as
    # the previous call returns), latency from arrival to return
    plain_open = {}
    for rate in (1000.0, 10000.0):
        to = workloads.Trace(1000 + rates.index(rate) if rate in rates else 77, 300, rate, VOLUME_DIMS, lods=4)
        plain_open[str(int(rate))] = plain_per_call(a, to, outs, device=True, arrivals=to.arrival_ns)
    a.close()
    # the reference's decoded-block cache (mc_cache_new_archive, 8 GiB) on the
    # same 400 requests, one at a time on the host
    ref_cache = reference_cache_trace(path, tr, args.q)
    os.remove(path)
    os.rmdir(td)
    return {"metric": "serving: p50/p99 request latency and GB/s of a Poisson block/region/chunk mix",
            "workload": "serve", "unit": "ms / GB/s", "n_gpus": 1, "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"serving over a {VOLUME_DIMS[2]}x{VOLUME_DIMS[1]}x{VOLUME_DIMS[0]} u8 volume, "
                                   f"LOD 0-3, q={args.q:g}, {nch} chunks",
                       "mix": "70% 16^3 blocks, 20% 128^3 regions, 10% 256^3 chunks",
                       "locality": "Zipf(1.1) over 128^3 cells", "cache": "8 GiB HBM decoded-block cache, S3-FIFO",
                       "classes": "requests up to 256 KiB of output batched on a high-priority stream, larger ones "
                                  "on a normal stream",
                       "outputs": "device memory", "batch_bytes": 512 << 20,
                       "archive_build_s": round(build_s, 2)},
            "rates": rows,
            "plain_per_call_device": plain_dev, "plain_per_call_host": plain_host,
            "plain_per_call_device_open_loop": plain_open,
            "reference_cache": ref_cache}


NAMES = ("block", "region", "chunk")


def _lat_summary(tr, lat, nbytes, seconds, api):
    lat = np.asarray(lat, np.float64)
    return {"api": api, "requests": len(tr), "p50_ms": round(pct(lat, 50), 4), "p99_ms": round(pct(lat, 99), 4),
            "p99_ms_by_kind": {NAMES[k]: round(pct(lat[tr.kind == k], 99), 4) for k in range(3) if (tr.kind == k).any()},
            "gbs": round(nbytes / seconds / 1e9, 3)}


def plain_per_call(a, tr, outs, device, arrivals=None):
    """The trace's requests one call at a time through the plain entry points:
    device outputs (mc_b200_read_regions_dev for blocks and regions,
    mc_b200_decode_chunks_dev for chunks; each call waits for its result) or
    host outputs (mc_archive_decode_block / read_region / decode_chunk).
    Closed loop by default (latency = the call); with arrival times (ns), each
    call starts at its arrival or when the previous one returns, and latency
    runs from the arrival. The first request of each kind runs once untimed
    before, so first-call allocations stay out of the latencies."""
    host = [np.zeros(n, np.uint8) for n in (4096, 128 ** 3, 256 ** 3)]   # pages touched
    lat, nbytes = [], 0

    def issue(i):
        k, lod = int(tr.kind[i]), int(tr.lod[i])
        z, y, x, dz, dy, dx = (int(v) for v in tr.req[i, :6])
        if device:
            if k == 0:
                a.read_regions_dev(lod, [(z * 16, y * 16, x * 16)], 16, 16, 16, outs[0].data_ptr())
            elif k == 1:
                a.read_regions_dev(lod, [(z, y, x)], dz, dy, dx, outs[1].data_ptr())
            else:
                a.decode_chunks_dev([a.chunk_offset(lod, z, y, x)], outs[2].data_ptr())
        else:
            if k == 0:
                co = a.chunk_offset(lod, z >> 4, y >> 4, x >> 4)
                if co > 1:
                    a.decode_block(co, z & 15, y & 15, x & 15)
            elif k == 1:
                a.read_region(lod, z, y, x, dz, dy, dx, out=host[1])
            else:
                a.decode_chunk(a.chunk_offset(lod, z, y, x), out=host[2])

    # untimed: the first request of each kind (first-call allocations)
    for kind in range(3):
        first = np.flatnonzero(tr.kind == kind)
        if first.size:
            issue(int(first[0]))
    t_all = time.perf_counter()
    for i in range(len(tr)):
        t1 = time.perf_counter()
        if arrivals is not None:
            t1 = t_all + float(arrivals[i]) / 1e9
            while time.perf_counter() < t1:
                pass
        issue(i)
        lat.append((time.perf_counter() - t1) * 1e3)
        nbytes += tr.out_bytes(i)
    secs = time.perf_counter() - t_all
    api = ("mc_b200_read_regions_dev / mc_b200_decode_chunks_dev (device outputs)" if device else
           "mc_archive_decode_block / read_region / decode_chunk (host outputs)")
    if arrivals is not None:
        api += f", open loop at {len(tr) / (float(arrivals[-1]) / 1e9):.0f} req/s offered"
        secs = max(secs, float(arrivals[-1]) / 1e9)
    return _lat_summary(tr, lat, nbytes, secs, api)


def reference_cache_trace(path, tr, q):
    """The reference's own mc_cache (8 GiB, bound to the archive) serving the
    trace one request at a time on the host (oracle/mc_cache_trace.c over the
    reference's default-flag build)."""
    from oracle import HERE as ORACLE_DIR
    lib_path = os.path.join(ORACLE_DIR, "_ref", "libmccachetrace.so")
    if not os.path.exists(lib_path):
        return {"unavailable": "oracle/_ref/libmccachetrace.so not built"}
    L = C.CDLL(lib_path)
    L.mcct_run.restype = C.c_int
    L.mcct_run.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_size_t, C.c_int, C.c_int,
                           C.c_void_p, C.c_void_p, C.c_void_p]
    n = len(tr)
    req = np.zeros((n, 8), np.int64)
    req[:, 0] = tr.kind
    req[:, 1] = tr.lod
    req[:, 2:8] = tr.req[:, :6]
    out = np.empty(256 ** 3, np.uint8)
    lat = np.zeros(n, np.float64)
    nz, ny, nx = VOLUME_DIMS
    t0 = time.perf_counter()
    rc = L.mcct_run(path.encode(), nx, ny, nz, q, 8 << 30, 0, n, req.ctypes.data, out.ctypes.data, lat.ctypes.data)
    secs = time.perf_counter() - t0
    if rc != 0:
        return {"unavailable": "mcct_run failed"}
    nbytes = sum(tr.out_bytes(i) for i in range(n))
    r = _lat_summary(tr, lat, nbytes, secs, "reference mc_cache_new_archive(8 GiB) + mc_cache_update / "
                                             "mc_cache_get_copy, one request at a time, host cores")
    r["cores"] = min(os.cpu_count() or 4, 16)
    return r


def run_regions(args):
    """Dataloader batch: 64 boxes of 128^3 at seeded random offsets with
    material fraction >= 0.5 into a strided u8 batch buffer (decode and crop
    fused), against the plain host read_regions and the reference's CPU."""
    import workloads
    from mcb200 import McLib
    lib = McLib.product()
    td = tempfile.mkdtemp()
    path = os.path.join(td, "regions.mca")
    a, nch = workloads.build_volume_archive(lib, path, VOLUME_DIMS, lods=8, q=args.q)
    t0 = time.perf_counter()
    boxes = a.sample_boxes(0, 20260101, 64, 128, 128, 128, 0.5)
    sample_host_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    boxes_dev = a.sample_boxes_dev(0, 20260101, 64, 128, 128, 128, 0.5)
    sample_dev_ms = (time.perf_counter() - t0) * 1e3
    sampling = {"api": "mc_b200_sample_boxes", "boxes": len(boxes), "ms": round(sample_dev_ms, 3),
                "host_call_ms": round(sample_host_ms, 3), "same_boxes_as_host_call": boxes_dev == boxes}
    crop = 128 ** 3
    stride = crop + 4096                        # strided batch: a 4 KiB gap between crops
    d_out = torch.zeros(stride * len(boxes), dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()   # a real stream: the library treats NULL as its own per-thread stream
    torch.cuda.set_stream(s)
    for _ in range(args.warmup):
        a.read_regions_dev(0, boxes, 128, 128, 128, d_out.data_ptr(), stride, s.cuda_stream)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for e0, e1 in ev:
        e0.record(s)
        a.read_regions_dev(0, boxes, 128, 128, 128, d_out.data_ptr(), stride, s.cuda_stream)
        e1.record(s)
    torch.cuda.synchronize()
    per_call_ms = statistics.median([e0.elapsed_time(e1) for e0, e1 in ev])
    dev = d_out.cpu().numpy()
    # the same batch as a graph-captured plan (work list, batch layout and
    # launch shape built once), replayed per step
    d_plan = torch.zeros_like(d_out)
    plan = a.plan_regions(0, boxes, 128, 128, 128, d_plan.data_ptr(), stride)
    plan_cfg = plan.tuning()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        plan.launch(s.cuda_stream)
    torch.cuda.synchronize()
    pt = []
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        plan.launch(s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize()
        pt.append(e0.elapsed_time(e1))
    ms = statistics.median(pt)
    plan_exact = bool(torch.equal(d_plan, d_out))
    _, plan_blocks, _ = plan.info()
    plan.free()
    del flush
    # plain drop-in, host output (warm: the median of 3 calls after one)
    host_ms, host = host_read_regions_ms(a, boxes, 128, 128, 128, stride)
    exact = bool(all(np.array_equal(dev[i * stride:i * stride + crop], host[i * stride:i * stride + crop])
                     for i in range(len(boxes))))
    # archive verification: chained XXH64 of every chunk blob of every LOD,
    # hashed on the device from the HBM mirror (the host walks the node tables)
    _, base, alen = a.sync_device()
    arc = np.fromfile(path, np.uint8)
    vt = []
    for _ in range(max(3, args.steps)):
        t0 = time.perf_counter()
        vbad = lib.L.mc_b200_verify_archive_dev(arc.ctypes.data, base, alen, 0)
        vt.append(time.perf_counter() - t0)
    verify = {"api": "mc_b200_verify_archive_dev", "archive_bytes": int(alen), "corrupt": int(vbad),
              "ms": round(statistics.median(vt[1:]) * 1e3, 3),
              "gbs": round(alen / statistics.median(vt[1:]) / 1e9, 3)}
    a.close()
    # parity against the reference's strict build (its default fast-math build
    # differs from itself under other flags by +-1 on about 1e-6 of voxels);
    # the timed CPU baseline is the default build
    exact_ref, cpu = None, None
    if not args.no_cpu_baseline:
        from oracle import REF_FAST_LIB, REF_LIB
        try:
            for lib_path, timed in ((REF_LIB, False), (REF_FAST_LIB, True)):
                ref = McLib(lib_path, b200=False)
                ref.L.mc_codec_init()
                with ref.open(path, VOLUME_DIMS[2], VOLUME_DIMS[1], VOLUME_DIMS[0], args.q) as ra:
                    if timed:   # the same warm timing as the host call above
                        ref_ms, rout = host_read_regions_ms(ra, boxes, 128, 128, 128, stride)
                        ref_s = ref_ms / 1e3
                    else:
                        rout = ra.read_regions(0, boxes, 128, 128, 128, batch_stride=stride)
                if timed:
                    t0 = time.perf_counter()
                    rbad = ref.L.mc_verify_archive(arc.ctypes.data, arc.size, 0)
                    verify["reference_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
                    verify["reference_corrupt"] = int(rbad)
                    verify["reference_api"] = "mc_verify_archive (one thread, the reference's default-flag build)"
                    cpu = {"value": round(len(boxes) * crop / ref_s / 1e9, 4), "unit": "GB/s",
                           "cores": min(os.cpu_count() or 4, 16), "kind": "reference",
                           "sample": "mc_archive_read_regions(nthreads=0) over the same 64 boxes, median of 3 "
                                     "calls after one into a touched buffer, the reference's default-flag build"}
                else:
                    exact_ref = bool(np.array_equal(rout, host))
        except (FileNotFoundError, OSError) as e:
            cpu = {"value": None, "sample": f"unavailable: {e}"}
    os.remove(path)
    os.rmdir(td)
    gb = len(boxes) * crop / 1e9
    return {"metric": "dataloader region batch: crop GB/s (64 x 128^3, strided batch)", "workload": "regions",
            "value": round(gb / (ms / 1e3), 3), "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "ms_per_step": round(ms, 4), "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"read_regions of 64 boxes of 128^3 (min material 0.5) from a "
                                   f"{VOLUME_DIMS[2]}x{VOLUME_DIMS[1]}x{VOLUME_DIMS[0]} u8 volume with 8 LODs at "
                                   f"q={args.q:g}, {nch} chunks, into a strided device batch",
                       "boxes": len(boxes), "batch_stride": stride},
            "bit_exact_device_vs_host_call": exact, "bit_exact_vs_reference_strict_build": exact_ref,
            "bit_exact_plan_vs_per_call": plan_exact,
            "api": "mc_b200_plan_read_regions + mc_b200_plan_launch (graph replay; L2 flushed between steps)",
            "launch_config": plan_cfg, "blocks_per_step": plan_blocks,
            "per_call": {"api": "mc_b200_read_regions_dev (work list built per call)", "ms": round(per_call_ms, 4),
                         "gbs": round(len(boxes) * crop / 1e9 / (per_call_ms / 1e3), 3)},
            "roofline": {"bound": "hbm", "achieved": round(len(boxes) * crop / 1e9 / (ms / 1e3), 3),
                         "peak": hbm_peak()[0], "peak_kind": hbm_peak()[1], "unit": "GB/s",
                         "frac": round(len(boxes) * crop / 1e9 / (ms / 1e3) / hbm_peak()[0], 4),
                         "algorithmic_bytes": "crop bytes written"},
            "plain_host_call": {"api": "mc_archive_read_regions (host output)", "ms": round(host_ms, 3),
                                "gbs": round(gb / (host_ms / 1e3), 3)},
            "verify": verify,
            "sampling": sampling,
            "cpu_baseline": cpu}


def run_deblock(args):
    """Decode-side deblocking of config 2's decoded chunks in HBM: the 64
    decoded 256^3 chunks, each deblocked as its own volume, in one
    mc_b200_deblock_dev call; the decoded bytes are restored before every
    step (a 1 GiB device copy, which also evicts the L2)."""
    from mcb200 import McLib
    lib = McLib.product()
    dev = torch.device("cuda", 0)
    vox = make_volumes(chunk_seeds(0, args.chunks), dev)
    td = tempfile.mkdtemp()
    path = os.path.join(td, "deblock.mca")
    a = lib.open(path, 256 * args.chunks, 256, 256, args.q)
    assert a.append_chunks(0, [(0, 0, c) for c in range(args.chunks)], [vox[c].data_ptr() for c in range(args.chunks)],
                           args.q, on_device=True) == 0
    del vox
    offs = [a.chunk_offset(0, 0, 0, c) for c in range(args.chunks)]
    dec = torch.empty(args.chunks * CHUNK, dtype=torch.uint8, device=dev)
    out = torch.empty_like(dec)
    plan = a.plan_chunks(offs, dec.data_ptr())
    # one non-default stream for every copy, decode and deblock: the library
    # treats a NULL stream as its own per-thread stream
    s = torch.cuda.Stream()
    torch.cuda.set_stream(s)
    plan.launch(s.cuda_stream)
    torch.cuda.synchronize()
    n = args.chunks

    def step():
        out.copy_(dec)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        assert lib.deblock_dev(out.data_ptr(), n, CHUNK, 256, 256, 256, args.q, s.cuda_stream) == 0
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)
    for _ in range(args.warmup):
        step()
    clocks = Clocks()
    clocks.start()
    times = [step() for _ in range(args.steps)]
    clk = clocks.stop()
    ms = statistics.median(times)
    # decode and deblock back to back (graph-captured decode, then the three deblock kernels)
    both = []
    for k in range(args.steps):
        out.fill_(k & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        plan.launch(s.cuda_stream)
        lib.deblock_dev(dec.data_ptr(), n, CHUNK, 256, 256, 256, args.q, s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize()
        both.append(e0.elapsed_time(e1))
    plan.launch(s.cuda_stream)   # dec: decoded voxels again
    step()                       # out: dec deblocked
    # exactness: the first and last chunk against the oracle's deblock of the same decoded voxels
    from oracle import Oracle
    orc = Oracle()
    exact = True
    for c in (0, n - 1):
        src = dec[c * CHUNK:(c + 1) * CHUNK].cpu().numpy().reshape(256, 256, 256)
        exact &= bool(np.array_equal(out[c * CHUNK:(c + 1) * CHUNK].cpu().numpy().reshape(256, 256, 256),
                                     orc.deblock(src.copy(), args.q)))
    # e2e: the drop-in mc_deblock on host chunks (host -> device -> host inside the call)
    host = torch.empty(CHUNK, dtype=torch.uint8).pin_memory().numpy()
    e2e = []
    for k in range(max(3, args.steps // 2)):
        host[:] = dec[(k % n) * CHUNK:(k % n + 1) * CHUNK].cpu().numpy()
        t0 = time.perf_counter()
        lib.deblock(host.reshape(256, 256, 256), args.q)
        e2e.append(time.perf_counter() - t0)
    e2e_gbs = CHUNK / statistics.median(e2e[1:]) / 1e9
    plan.free()
    a.close()
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import REF_FAST_LIB
        try:
            import ctypes as C
            R = C.CDLL(REF_FAST_LIB)
            R.mc_deblock.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
            k, t_cpu = 0, 0.0
            while t_cpu < 8.0 and k < n:
                buf = np.zeros(CHUNK + 256 * 256, np.uint8)
                buf[:CHUNK] = dec[k * CHUNK:(k + 1) * CHUNK].cpu().numpy()
                t0 = time.perf_counter()
                R.mc_deblock(buf.ctypes.data, 256, 256, 256, args.q)
                t_cpu += time.perf_counter() - t0
                k += 1
            cpu = {"value": round(k * CHUNK / t_cpu / 1e9, 4), "unit": "GB/s", "cores": 1, "kind": "reference",
                   "sample": f"the reference's mc_deblock (single-threaded, default-flag build) on {k} of the "
                             f"same decoded 256^3 chunks"}
        except (FileNotFoundError, OSError) as e:
            cpu = {"value": None, "sample": f"unavailable: {e}"}
    os.remove(path)
    os.rmdir(td)
    peak, peak_kind = hbm_peak()
    vol = n * CHUNK
    achieved = 2 * vol / (ms / 1e3) / 1e9
    return {"metric": "deblocked GB/s of decoded volume (mc_deblock on device)", "workload": "deblock",
            "value": round(vol / (ms / 1e3) / 1e9, 3), "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "dtype": "u8",
            "data": "synthetic", "vs_baseline": None,
            "config": {"workload": f"deblock {n} decoded 256^3 chunks (config 2 volumes, q={args.q:g}) in HBM, one "
                                   f"volume per chunk, quality {args.q:g}",
                       "l2": "1 GiB device copy before every step"},
            "gpu_launches": 3 * args.steps,
            "bit_exact_vs_oracle": exact,
            "decode_and_deblock_gbs": round(vol / (statistics.median(both) / 1e3) / 1e9, 3),
            "e2e": {"value": round(e2e_gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": CHUNK,
                    "d2h_bytes_per_step": CHUNK, "api": "mc_deblock (host volume, one 256^3 chunk per call)"},
            "roofline": {"bound": "hbm", "kernel": "k_deblock_x + k_deblock_y + k_deblock_z",
                         "achieved": round(achieved, 2), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None,
                         "algorithmic_bytes_per_launch": 2 * vol},
            "clocks": clk, "cpu_baseline": cpu}


def _blob_len(data, co):
    """Length of the chunk blob at byte offset co of archive bytes."""
    fml = data[co + 12] | (data[co + 13] << 8)
    bm = np.frombuffer(data[co + 14 + fml:co + 14 + fml + 512], np.uint8)
    npres = int(np.unpackbits(bm).sum())
    lens = np.frombuffer(data[co + 14 + fml + 512:co + 14 + fml + 512 + 2 * npres], np.uint16)
    return 14 + fml + 512 + 2 * npres + int(lens.astype(np.int64).sum())


def _pyramid_levels(nz, ny, nx):
    """The one-shot builder's LOD loop (src/mc_archive.c:205-220): [(lod, padded extent)]."""
    d = tuple((n + 255) // 256 * 256 for n in (nz, ny, nx))
    out = []
    for lod in range(8):
        if min(d) < 1 or not (max(d) >= 256 or lod == 0):
            break
        out.append((lod, d))
        if min(v // 2 for v in d) < 1 or (max(v // 2 for v in d) < 256 and lod >= 1):
            break
        d = tuple((v + 1) // 2 for v in d)
    return out


def _mc_build(lib_path, vol, q):
    """The reference's one-shot builder (mc_build) over a host volume, through
    the oracle's buffer voxel source; returns (archive bytes, seconds)."""
    import ctypes as C
    from oracle import ORACLE_LIB

    class Opts(C.Structure):
        _fields_ = [("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("quality", C.c_float),
                    ("metadata", C.c_char_p), ("meta_len", C.c_size_t)]

    class Src(C.Structure):
        _fields_ = [("v", C.c_void_p), ("nz", C.c_int), ("ny", C.c_int), ("nx", C.c_int)]
    R, O = C.CDLL(lib_path), C.CDLL(ORACLE_LIB)
    R.mc_codec_init()
    R.mc_build.restype = C.c_void_p
    R.mc_build.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_size_t)]
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    vol = np.ascontiguousarray(vol)
    nz, ny, nx = vol.shape
    src, opts, n = Src(vol.ctypes.data, nz, ny, nx), Opts(0, nx, ny, nz, q, None, 0), C.c_size_t()
    t0 = time.perf_counter()
    buf = R.mc_build(C.cast(O.or_voxel_source, C.c_void_p), C.byref(src), C.byref(opts), C.byref(n))
    dt = time.perf_counter() - t0
    data = C.string_at(buf, n.value)
    libc.free(buf)
    return data, dt


def run_pyramid(args):
    """LOD pyramid build: a 1024^3 u8 volume resident in HBM appended with all
    its LODs (decimated on the device, encoded by the batched encoder, installed
    in the archive file) by one mc_b200_append_pyramid call per step."""
    from mcb200 import McLib
    import volumes
    lib = McLib.product()
    dims = (1024, 1024, 1024)
    vol = volumes.region(7, (0, 0, 0), dims, 0.4, device="cuda").contiguous()
    td = tempfile.mkdtemp()
    times, nl, chunks, arc_bytes = [], 0, 0, 0
    for k in range(args.warmup + args.steps):
        path = os.path.join(td, f"pyr{k}.mca")
        with lib.open(path, dims[2], dims[1], dims[0], args.q) as a:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rc, nl = a.append_pyramid(vol.data_ptr(), *dims, args.q)
            dt = time.perf_counter() - t0
            assert rc == 0
            arc_bytes = int(a.L.mc_archive_data_len(a.a))
        os.remove(path)
        if k >= args.warmup:
            times.append(dt)
    s = statistics.median(times)
    # exactness and the CPU baseline on a 512^3 sample of the same volume: the
    # device pyramid's chunk blobs against the reference builder's
    sample = vol[:512, :512, :512].contiguous()
    h = sample.cpu().numpy()
    exact, cpu = None, None
    if not args.no_cpu_baseline:
        from oracle import REF_FAST_LIB, REF_LIB
        try:
            ref_data, _ = _mc_build(REF_LIB, h, args.q)
            _, cpu_s = _mc_build(REF_FAST_LIB, h, args.q)
            path = os.path.join(td, "sample.mca")
            rpath = os.path.join(td, "ref.mca")
            open(rpath, "wb").write(ref_data)
            ref = McLib(REF_LIB, b200=False)
            ref.L.mc_codec_init()
            exact = True
            with lib.open(path, 512, 512, 512, args.q) as a, ref.open(rpath, 512, 512, 512, args.q) as ra:
                assert a.append_pyramid(sample.data_ptr(), 512, 512, 512, args.q)[0] == 0
                mine = open(path, "rb").read()
                for lod, (dz, dy, dx) in _pyramid_levels(512, 512, 512):
                    for c in range(((dz + 255) // 256) * ((dy + 255) // 256) * ((dx + 255) // 256)):
                        nc = ((dy + 255) // 256, (dx + 255) // 256)
                        cz, cy, cx = c // (nc[0] * nc[1]), (c // nc[1]) % nc[0], c % nc[1]
                        o1, o2 = a.chunk_offset(lod, cz, cy, cx), ra.chunk_offset(lod, cz, cy, cx)
                        b1 = mine[o1:o1 + _blob_len(mine, o1)] if o1 > 1 else b""
                        b2 = ref_data[o2:o2 + _blob_len(ref_data, o2)] if o2 > 1 else b""
                        exact &= b1 == b2
            os.remove(path)
            os.remove(rpath)
            cpu = {"value": round(h.size / cpu_s / 1e9, 4), "unit": "GB/s of LOD-0 voxels", "cores": 1,
                   "kind": "reference",
                   "sample": "the reference's mc_build (one thread, default-flag build) over a 512^3 sample of the "
                             "same volume: LOD 0 and LOD 1"}
        except (FileNotFoundError, OSError) as e:
            cpu = {"value": None, "sample": f"unavailable: {e}"}
    os.rmdir(td)
    vbytes = dims[0] * dims[1] * dims[2]
    return {"metric": "LOD pyramid build: GB/s of LOD-0 voxels (decimate + encode + install)", "workload": "pyramid",
            "value": round(vbytes / s / 1e9, 3), "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(s * 1e3, 2), "higher_is_better": True, "dtype": "u8",
            "data": "synthetic", "vs_baseline": None,
            "config": {"workload": f"mc_b200_append_pyramid of a 1024^3 u8 volume (40 % air) in HBM at q={args.q:g}: "
                                   f"{nl} LODs into a new archive file per step"},
            "archive_bytes": arc_bytes, "bit_exact_vs_reference_builder_on_sample": exact, "cpu_baseline": cpu}


def run_encode(args):
    """Preset ladder: 8 chunks (30 % air) encoded at each of the 8 presets
    (q and tau from the preset table) in one batched append per level."""
    from mcb200 import McLib
    import volumes
    lib = McLib.product()
    vox = [volumes.region(s, (0, 0, 256 * s), (256, 256, 256), 0.3, device="cuda").contiguous() for s in range(8)]
    td = tempfile.mkdtemp()
    rows, worst = [], 0
    for lvl in range(8):
        q, tau = float(lib.L.mc_preset_quality(lvl)), int(lib.L.mc_preset_tau(lvl))
        path = os.path.join(td, f"enc{lvl}.mca")
        times = []
        for rep in range(max(1, args.steps // 2) + 1):
            with lib.open(path + f".{rep}", 256 * 8, 256, 256, q) as a:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                rc = a.append_chunks(0, [(0, 0, c) for c in range(8)], [v.data_ptr() for v in vox], q, ctx_q=q,
                                     ctx_tau=tau, on_device=True)
                times.append(time.perf_counter() - t0)
                assert rc == 0
                if rep == 0:
                    dec = a.decode_chunk(a.chunk_offset(0, 0, 0, 3)).reshape(256, 256, 256)
                    err = int(np.abs(dec.astype(int) - vox[3].cpu().numpy().astype(int)).max())
                    worst = max(worst, err - tau)
                size = int(a.L.mc_archive_data_len(a.a))
            os.remove(path + f".{rep}")
        t = statistics.median(times[1:]) if len(times) > 1 else times[0]
        rows.append({"level": lvl, "q": q, "tau": tau, "gbs": round(8 * CHUNK / t / 1e9, 3), "ms": round(t * 1e3, 2),
                     "archive_bytes": size})
    # the reference's own encode of the same chunks at preset 4 (q=6, tau=16):
    # its ctx path (one thread) and its parallel path (all threads, no tau)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import REF_FAST_LIB
        try:
            ref = McLib(REF_FAST_LIB, b200=False)
            ref.L.mc_codec_init()
            host = [v.cpu().numpy() for v in vox[:2]]
            res = {}
            for mode in ("ctx", "par"):
                path = os.path.join(td, f"ref_{mode}.mca")
                with ref.open(path, 256 * 8, 256, 256, 6.0) as a:
                    c = ref.ctx(6.0, 16)
                    t0 = time.perf_counter()
                    for i, h in enumerate(host):
                        if mode == "ctx":
                            assert ref.L.mc_archive_append_chunk_ctx(a.a, c, 0, 0, 0, i, h.ctypes.data) == 0
                        else:
                            assert ref.L.mc_archive_append_chunk_par(a.a, 0, 0, 0, i, h.ctypes.data, 6.0, 0) == 0
                    res[mode] = len(host) * CHUNK / (time.perf_counter() - t0) / 1e9
                    ref.L.mc_codec_ctx_free(c)
                os.remove(path)
            cpu = {"value": round(res["ctx"], 4), "unit": "GB/s", "cores": 1, "kind": "reference",
                   "sample": "the reference's mc_archive_append_chunk_ctx at preset 4 (q=6, tau=16) on 2 of the "
                             "same chunks, default-flag build",
                   "parallel_path_gbs": round(res["par"], 4),
                   "parallel_path": f"mc_archive_append_chunk_par(nthreads=0, q=6, no tau) on {os.cpu_count()} "
                                    "host threads"}
        except (FileNotFoundError, OSError) as e:
            cpu = {"value": None, "sample": f"unavailable: {e}"}
    os.rmdir(td)
    return {"metric": "preset-ladder batched encode: raw GB/s per level (8 x 256^3, 30% air)",
            "workload": "encode", "unit": "GB/s", "n_gpus": 1, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "mc_b200_append_chunks of 8 chunks per preset level (q, tau from the preset "
                                   "table), host timing around the call (encode, blob assembly, install)"},
            "levels": rows, "tau_bound_holds": worst <= 0, "cpu_baseline": cpu}

# ------------------------------------------------------------------ arms
def run_reference(args, d):
    if d.rank != 0:
        return None
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    vox = make_volumes(chunk_seeds(0, args.chunks), dev).cpu().numpy()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "ref.mca")
        build_reference_archive(path, vox, args.q)
        gbs, cores, done, times = reference_decode(path, args.chunks, args.q, args.steps, args.warmup)
    ms = statistics.mean(times) * 1e3
    sample = f"mc_archive_decode_chunk(nthreads=0) over all {args.chunks} chunks, {done} steps"
    return {"metric": METRIC, "value": round(gbs, 4), "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": done, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": config(args, 1),
            "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_b200(args, d):
    from mcb200 import McLib, decode_chunk_blobs
    lib = McLib.product()
    # each rank's library runs on the rank's own GPU (its current device, set
    # before any CUDA work): a rank bound elsewhere would time the wrong GPU
    if lib.L.mc_b200_device() != torch.cuda.current_device():
        raise RuntimeError(f"rank {d.rank}: library on device {lib.L.mc_b200_device()}, "
                           f"torch on device {torch.cuda.current_device()}")
    dev = torch.device("cuda", torch.cuda.current_device())
    seeds = chunk_seeds(d.rank, args.chunks)
    vox = make_volumes(seeds, dev)
    td = tempfile.mkdtemp()
    path = os.path.join(td, f"bench_{d.rank}.mca")
    a = lib.open(path, 256 * args.chunks, 256, 256, args.q)
    rc = a.append_chunks(0, [(0, 0, c) for c in range(args.chunks)], [vox[c].data_ptr() for c in range(args.chunks)],
                         args.q, on_device=True)
    assert rc == 0, "append failed"
    del vox
    offs = [a.chunk_offset(0, 0, 0, c) for c in range(args.chunks)]
    out = torch.empty(args.chunks * CHUNK, dtype=torch.uint8, device=dev)
    plan = a.plan_chunks(offs, out.data_ptr())
    launches_per_step, blocks, payload = plan.info()
    plan_cfg = plan.tuning()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream()
    for w in range(args.warmup):
        flush.fill_(w & 0xFF)
        plan.launch(s.cuda_stream)
    torch.cuda.synchronize()
    d.barrier()
    torch.cuda.synchronize()
    clocks = Clocks()
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(s)
        plan.launch(s.cuda_stream)
        ev[k][1].record(s)
    torch.cuda.synchronize()
    clk = clocks.stop()
    d.barrier()
    torch.cuda.synchronize()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    ms = d.max(sum(step_ms)) / args.steps
    decoded = d.world * args.chunks * CHUNK
    value = decoded / (ms / 1e3) / 1e9

    # per-stage timing: each kernel alone on the same stream, CUDA events (the
    # NVTX range lets a profiler pick these launches, at the tuned shapes)
    stage_ms = [0.0, 0.0]
    torch.cuda.nvtx.range_push("stages")
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        for stage in (0, 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            plan.launch_stage(stage, s.cuda_stream)
            e1.record(s)
            torch.cuda.synchronize()
            stage_ms[stage] += e0.elapsed_time(e1) / args.steps
    torch.cuda.nvtx.range_pop()

    # the whole decode under each stage layout the autotuner chose among,
    # its entropy and reconstruction shapes kept (the chosen layout is the step above)
    layout_ms = {}
    tuned = [plan_cfg[k] for k in ("entropy_warps_per_cta", "entropy_ctas_per_sm", "entropy_claim",
                                   "reconstruct_ctas_per_sm")]
    solo = plan_cfg["entropy_solo_share"]
    for stages in plan.STAGES:
        if plan.set_tuning(*tuned, stages, solo) != 0:
            continue
        for k in range(2):
            plan.launch(s.cuda_stream)
        tot = 0.0
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            plan.launch(s.cuda_stream)
            e1.record(s)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        layout_ms[stages] = round(tot / args.steps, 4)
    plan.set_tuning(*tuned, plan_cfg["stages"], solo)
    plan.launch(s.cuda_stream)
    torch.cuda.synchronize()

    # bit-exactness spot check against the oracle on one chunk (rank 0)
    exact = None
    if d.rank == 0:
        from oracle import Oracle
        blob = bytes(blobs_of(path, [offs[0]])[0])
        exact = bool(np.array_equal(out[:CHUNK].cpu().numpy(), Oracle().decode_chunk(blob)))

    # plain per-call drop-in latency: mc_archive_decode_block on random blocks
    # (the reference's own decode_block times the same blocks below)
    rng = np.random.Generator(np.random.PCG64(d.rank))
    picks = [(int(rng.integers(0, args.chunks)), int(rng.integers(0, 4096))) for _ in range(320)]
    lat = block_latency(a, offs, picks)
    # config 1's plain method: all 4096 blocks of one chunk, one decode_block call each
    plain_ms = plain_chunk_blocks_ms(a, offs[0])

    # e2e: host blobs (pinned) -> host voxels (pinned) through the C ABI
    blobs = blobs_of(path, offs)
    pinned = [torch.from_numpy(b).pin_memory().numpy() for b in blobs]
    hout = torch.empty(args.chunks * CHUNK, dtype=torch.uint8).pin_memory().numpy()
    h2d = int(sum(b.size for b in pinned))
    for _ in range(max(1, args.warmup // 2)):
        decode_chunk_blobs(lib, pinned, hout)
    d.barrier()
    e2e_s = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        decode_chunk_blobs(lib, pinned, hout)
        e2e_s.append(time.perf_counter() - t0)
    e2e_value = decoded / (d.max(sum(e2e_s)) / args.steps) / 1e9
    e2e_exact = bool(np.array_equal(hout[:CHUNK], out[:CHUNK].cpu().numpy())) if d.rank == 0 else None
    # the link bound of e2e: one plain pinned device-to-host copy of the same voxels
    hview = torch.from_numpy(hout)
    cs = torch.cuda.Stream()
    with torch.cuda.stream(cs):
        hview.copy_(out, non_blocking=True)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(cs)
        for _ in range(3):
            hview.copy_(out, non_blocking=True)
        ev1.record(cs)
    ev1.synchronize()
    d2h_gbs = 3 * args.chunks * CHUNK / (ev0.elapsed_time(ev1) / 1e3) / 1e9

    plan.free()
    a.close()

    ref_lat = ref_plain_ms = None
    if d.rank == 0 and d.world == 1 and not args.no_cpu_baseline:
        try:
            ref_lat, ref_plain_ms = reference_block_latency(path, args.chunks, args.q, picks)
        except (FileNotFoundError, OSError):
            pass
    cpu = None
    if d.rank == 0 and d.world == 1 and not args.no_cpu_baseline:
        try:
            gbs, cores, done, _ = reference_decode(path, args.chunks, args.q, 100, 1, min_seconds=8.0)
            cpu = {"value": round(gbs, 4), "unit": "GB/s", "cores": cores, "kind": "reference",
                   "sample": f"reference mc_archive_decode_chunk(nthreads=0) over the same {args.chunks}-chunk "
                             f"archive, {done} passes (~8 s), sources built with the reference's default flags"}
        except (FileNotFoundError, OSError) as e:
            cpu = {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}
    os.remove(path)
    os.rmdir(td)
    if d.rank != 0:
        return None

    peak, peak_kind = hbm_peak()
    ent_ms = stage_ms[0]
    achieved = args.chunks * CHUNK / (ent_ms / 1e3) / 1e9
    traffic = (ENTROPY_DRAM_BYTES_PER_CHUNK * args.chunks) if ENTROPY_DRAM_BYTES_PER_CHUNK else None
    return {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": d.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded value-noise volumes; the reference's scroll CT data is not available offline)",
        "config": config(args, d.world),
        "gpu_launches": launches_per_step * args.steps,
        "bit_exact_vs_oracle": exact,
        "e2e": {"value": round(e2e_value, 3), "unit": "GB/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": args.chunks * CHUNK, "api": "mc_b200_decode_chunk_blobs",
                "bit_exact": e2e_exact, "d2h_copy_gbs": round(d2h_gbs, 2),
                "d2h_copy": "plain pinned device-to-host copy of the same voxels (the PCIe bound of e2e)"},
        "roofline": {"bound": "hbm", "kernel": "k_entropy (entropy decode stage)", "achieved": round(achieved, 2),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic, "algorithmic_bytes_per_launch": args.chunks * CHUNK,
                     "kernel_ms": round(ent_ms, 4), "reconstruct_ms": round(stage_ms[1], 4),
                     "step_frac": round(value / d.world / peak, 4)},
        "latency": {"api": "mc_archive_decode_block (plain per-call drop-in, host buffer), 300 random blocks",
                    "p50_ms": round(pct(lat, 50), 4), "p99_ms": round(pct(lat, 99), 4),
                    "reference_p50_ms": None if ref_lat is None else round(pct(ref_lat, 50), 4),
                    "reference_p99_ms": None if ref_lat is None else round(pct(ref_lat, 99), 4),
                    "reference": "the reference's own mc_archive_decode_block (default-flag build, one host thread) "
                                 "on the same blocks of the same archive file"},
        "plain_chunk_decode": {"what": "4096 x mc_archive_decode_block over one 256^3 chunk (config 1's plain method)",
                               "gpu_ms": round(plain_ms, 3), "gpu_gbs": round(CHUNK / plain_ms / 1e6, 4),
                               "reference_ms": None if ref_plain_ms is None else round(ref_plain_ms, 3),
                               "reference_gbs": None if ref_plain_ms is None else round(CHUNK / ref_plain_ms / 1e6, 4)},
        "blocks_per_step": blocks, "payload_bytes_per_step": payload, "launch_config": plan_cfg,
        "stage_layout_ms": layout_ms,
        "clocks": clk,
        "cpu_baseline": cpu,
    }


def main():
    args = parse()
    d = Dist("nccl" if torch.cuda.is_available() else "gloo")
    try:
        if args.workload != "decode":
            if d.world > 1:
                raise SystemExit("the serve / regions / encode / deblock / pyramid workloads run on one GPU")
            res = {"serve": run_serve, "regions": run_regions, "encode": run_encode,
                   "deblock": run_deblock, "pyramid": run_pyramid}[args.workload](args)
        elif args.q_sweep:
            for q in (1.0, 3.0, 6.0, 12.0):
                args.q = q
                res = run_reference(args, d) if args.impl == "reference" else run_b200(args, d)
                if res is not None:
                    print(json.dumps(res), flush=True)
                torch.cuda.empty_cache()
            res = None
        else:
            res = run_reference(args, d) if args.impl == "reference" else run_b200(args, d)
        if res is not None:
            print(json.dumps(res), flush=True)
    finally:
        d.close()


if __name__ == "__main__":
    main()
