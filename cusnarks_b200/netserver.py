"""TCP front end with the reference prove server's protocol, over the continuous-batching server.

    python -m cusnarks_b200.netserver --pk circuit_pk.bin [--port 8192] [--slots 3]

Protocol of src/python/groth_prover.py:808-891 startServer with src/python/json_socket.py
framing (a native uint32 byte count, then JSON text):
  {"is_alive": 1}                       -> {"status": 1}
  {"witness_f": w, "proof_f": p, "public_data_f": q, "verify_en": v}
                                        -> queued; the proof is written to p and the public
                                           signals to q when done (no reply, as the reference)
  {"list": k}                           -> the k-th request record (witness_f, proof_f,
                                           public_data_f, verify_en, proof_id, result, and
                                           latency_ms); result -1 while pending, 1 written,
                                           0 failed
  {"stop_server": 1}                    -> stops
Differences: requests that arrive while proofs run are admitted (continuous batching)
instead of dropped; verify_en is recorded but no verification runs (the reference shells
out to snarkjs).  Proof files: `.json` (pi_a, pi_b, pi_c in normal form as decimal strings,
"protocol": "groth", write_proof :1705) or `.bin` (normal-form words pi_a | pi_b | pi_c).
"""
from __future__ import annotations

import argparse
import json
import socket
import struct
import threading

import numpy as np

from . import pkfile

Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R_INV_Q = pow(1 << 256, -1, Q)


def _int(words) -> int:
    return sum(int(x) << (32 * i) for i, x in enumerate(words))


def proof_to_json(proof: np.ndarray) -> dict:
    """64 words (affine Montgomery pi_A | pi_B | pi_C) -> the reference's proof.json fields."""
    v = [(_int(proof[8 * i:8 * i + 8]) * R_INV_Q) % Q for i in range(8)]
    return {"pi_a": [str(v[0]), str(v[1]), "1"],
            "pi_b": [[str(v[2]), str(v[3])], [str(v[4]), str(v[5])], ["1", "0"]],
            "pi_c": [str(v[6]), str(v[7]), "1"],
            "protocol": "groth"}


def proof_to_words(proof: np.ndarray) -> np.ndarray:
    v = [(_int(proof[8 * i:8 * i + 8]) * R_INV_Q) % Q for i in range(8)]
    return np.concatenate([[(x >> (32 * k)) & 0xffffffff for k in range(8)] for x in v]).astype(np.uint32)


def recv_msg(conn) -> dict | None:
    head = b""
    while len(head) < 4:
        chunk = conn.recv(4 - len(head))
        if not chunk:
            return None
        head += chunk
    n = struct.unpack("I", head)[0]
    body = b""
    while len(body) < n:
        chunk = conn.recv(min(65536, n - len(body)))
        if not chunk:
            return None
        body += chunk
    return json.loads(body.decode())


def send_msg(conn, data: dict):
    text = json.dumps(data, indent=2).encode()
    conn.sendall(struct.pack("I", len(text)) + text)


class NetProveServer:
    """Socket front end: one listener thread, one completion thread, the C++ server under them."""

    def __init__(self, prover, n_public: int, host: str = "127.0.0.1", port: int = 8192, slots: int = 3,
                 device: int = 0):
        from .server import ProveServer
        self.srv = ProveServer(device, slots=slots)
        self.key = self.srv.add_key(prover)
        self.n_vars = prover.n_vars
        self.n_public = n_public
        self.repo = []
        self.lock = threading.Lock()
        self.pending = []
        self.cv = threading.Condition(self.lock)
        self.sock = socket.socket(socket.AF_INET, socket.SOCK_STREAM)
        self.sock.setsockopt(socket.SOL_SOCKET, socket.SO_REUSEADDR, 1)
        self.sock.bind((host, port))
        self.sock.listen(16)
        self.port = self.sock.getsockname()[1]
        self.stopped = threading.Event()
        self.t_listen = threading.Thread(target=self._listen, daemon=True)
        self.t_done = threading.Thread(target=self._complete, daemon=True)
        self.t_listen.start()
        self.t_done.start()

    # requests ---------------------------------------------------------------------------
    def _submit(self, msg: dict):
        rec = {"witness_f": msg["witness_f"], "proof_f": msg.get("proof_f"),
               "public_data_f": msg.get("public_data_f"), "verify_en": int(msg.get("verify_en", 0)),
               "result": -1}
        with self.lock:
            rec["proof_id"] = len(self.repo)
            self.repo.append(rec)
        try:
            w = pkfile.read_witness(rec["witness_f"], self.n_vars)
            r = np.frombuffer(np.random.default_rng().bytes(32), dtype=np.uint32).copy()
            s = np.frombuffer(np.random.default_rng().bytes(32), dtype=np.uint32).copy()
            r[7] &= 0x0fffffff
            s[7] &= 0x0fffffff
            t = self.srv.submit(self.key, w, r, s)
        except Exception as e:  # unreadable witness: record the failure
            with self.lock:
                rec["result"], rec["error"] = 0, str(e)
            return
        with self.cv:
            self.pending.append((t, rec, w))
            self.cv.notify()

    def _complete(self):
        while not self.stopped.is_set():
            with self.cv:
                while not self.pending and not self.stopped.is_set():
                    self.cv.wait(0.2)
                if self.stopped.is_set():
                    return
                t, rec, w = self.pending.pop(0)
            try:
                proof, info = self.srv.wait(t)
                self._write(rec, proof, w)
                res, extra = 1, {"latency_ms": round(info["latency_ms"], 3)}
            except Exception as e:
                res, extra = 0, {"error": str(e)}
            with self.lock:
                rec["result"] = res
                rec.update(extra)

    def _write(self, rec, proof, w):
        pf, qf = rec["proof_f"], rec["public_data_f"]
        if pf:
            if str(pf).endswith(".bin"):
                proof_to_words(proof).astype("<u4").tofile(pf)
            else:
                with open(pf, "w") as f:
                    print(json.dumps(proof_to_json(proof), indent=4, sort_keys=True), file=f)
        if qf:
            pub = w[1:self.n_public + 1]
            if str(qf).endswith(".bin"):
                np.concatenate([[pub.shape[0]], pub.reshape(-1)]).astype("<u4").tofile(qf)
            else:
                with open(qf, "w") as f:
                    print(json.dumps([str(_int(row)) for row in pub], indent=4), file=f)

    # socket -----------------------------------------------------------------------------
    def _listen(self):
        while not self.stopped.is_set():
            try:
                conn, _ = self.sock.accept()
            except OSError:
                return
            with conn:
                try:
                    msg = recv_msg(conn)
                except (OSError, ValueError):
                    continue
                if not msg:
                    continue
                if msg.get("stop_server") == 1:
                    self.stopped.set()
                    with self.cv:
                        self.cv.notify_all()
                    self.sock.close()
                    return
                if "is_alive" in msg:
                    send_msg(conn, {"status": 1})
                elif "list" in msg:
                    k = int(msg["list"])
                    with self.lock:
                        if -len(self.repo) <= k < len(self.repo):
                            send_msg(conn, dict(self.repo[k]))
                        else:
                            send_msg(conn, {})
                elif "witness_f" in msg:
                    self._submit(msg)

    def close(self):
        if not self.stopped.is_set():
            self.stopped.set()
            try:
                self.sock.close()
            except OSError:
                pass
        with self.cv:
            self.cv.notify_all()
        self.t_done.join(timeout=30)
        self.srv.close()


def request(port: int, msg: dict, host: str = "127.0.0.1", reply: bool = True):
    """Client helper: send one message, return the reply dict (or None)."""
    with socket.create_connection((host, port), timeout=30) as c:
        send_msg(c, msg)
        return recv_msg(c) if reply else None


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m cusnarks_b200.netserver")
    ap.add_argument("--pk", required=True, help="proving key .bin (reference format)")
    ap.add_argument("--port", type=int, default=8192)
    ap.add_argument("--host", default="127.0.0.1")
    ap.add_argument("--slots", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    from .context import Context
    from .groth import Prover
    ctx = Context(args.device)
    pk = pkfile.read_pk_bin(args.pk, ctx)
    prover = Prover(ctx, pk)
    s = NetProveServer(prover, pk["n_public"], args.host, args.port, args.slots, args.device)
    print(f"listening on {args.host}:{s.port}", flush=True)
    s.stopped.wait()
    s.close()
    prover.close()


if __name__ == "__main__":
    main()
