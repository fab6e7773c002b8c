"""A PostgreSQL v3 wire-protocol front-end (simple query) for the serving loop.

It speaks the part of the protocol the reference's server uses for a read-only
SELECT (src/server/pgwire.rs): the startup packet (SSLRequest answered 'N'),
AuthenticationOk, ParameterStatus, BackendKeyData, ReadyForQuery; then per
'Q' message every ';'-separated statement is answered with RowDescription
('T', text format, INT8 / FLOAT8 / TEXT type OIDs), DataRow ('D') per row and
CommandComplete ('C', "SELECT n"), or ErrorResponse ('E', severity, SQLSTATE,
message) — after which the rest of the message is skipped — and the message
ends with ReadyForQuery ('Z', 'I'); 'S' (Sync) answers ReadyForQuery, 'X'
closes, any other message gets ErrorResponse 0A000 (pgwire.rs:99-160,
238-270, 438-524, 844-990).

Each connection runs on its own thread and hands statements to an executor
(``execute(sql) -> (column names, rows of text)``, raising ``SqlError``). The
reference runs a read-only SELECT under its engine's read lock and anything
else under the write lock (pgwire.rs:485-499); here the executor is either the
plain one-statement-at-a-time path or the continuous-batching serving loop
(``turbogp_b200.frontend``), and connections never block one another while
their statements wait for the GPU.

``PgWireClient`` is a minimal client of the same protocol (for the benchmark
and the tests).
"""
from __future__ import annotations

import os
import socket
import struct
import threading

from .sqlfront import SqlError

PROTOCOL_V3 = 196608
SSL_REQUEST = 80877103
CANCEL_REQUEST = 80877102
OID_INT8, OID_FLOAT8, OID_TEXT = 20, 701, 25


def _msg(kind: bytes, body: bytes = b"") -> bytes:
    return kind + struct.pack("!i", len(body) + 4) + body


def _cstr(s: str) -> bytes:
    return s.encode("utf-8") + b"\x00"


def _recv_exact(sock: socket.socket, n: int) -> bytes:
    buf = bytearray()
    while len(buf) < n:
        chunk = sock.recv(n - len(buf))
        if not chunk:
            raise EOFError("connection closed")
        buf += chunk
    return bytes(buf)


def error_response(sqlstate: str, message: str) -> bytes:
    body = b"S" + _cstr("ERROR") + b"V" + _cstr("ERROR") + b"C" + _cstr(sqlstate) + b"M" + _cstr(message) + b"\x00"
    return _msg(b"E", body)


def _type_oid(values: list[str]) -> int:
    """INT8 when every value of the column is an integer, FLOAT8 when every
    value is a number, else TEXT (the reference falls back the same way,
    pgwire.rs:852-872)."""
    if all(v.lstrip("-").isdigit() for v in values):
        return OID_INT8
    try:
        for v in values:
            float(v)
        return OID_FLOAT8
    except ValueError:
        return OID_TEXT


def result_messages(names: list[str], rows: list[tuple]) -> bytes:
    out = bytearray()
    body = bytearray(struct.pack("!h", len(names)))
    for j, name in enumerate(names):
        oid = _type_oid([r[j] for r in rows]) if rows else OID_INT8
        size = -1 if oid == OID_TEXT else 8
        body += _cstr(name) + struct.pack("!ihihih", 0, 0, oid, size, -1, 0)
    out += _msg(b"T", bytes(body))
    for r in rows:
        body = bytearray(struct.pack("!h", len(r)))
        for v in r:
            b = str(v).encode("utf-8")
            body += struct.pack("!i", len(b)) + b
        out += _msg(b"D", bytes(body))
    out += _msg(b"C", _cstr(f"SELECT {len(rows)}"))
    return bytes(out)


def split_statements(sql: str) -> list[str]:
    return [s.strip() for s in sql.split(";") if s.strip()]


class PgWireServer:
    """Accepts connections on (host, port) (port 0 = any free port) and
    serves each on its own thread until stop()."""

    PARAMS = (("server_version", "15.0"), ("server_encoding", "UTF8"), ("client_encoding", "UTF8"),
              ("DateStyle", "ISO, MDY"), ("integer_datetimes", "on"), ("standard_conforming_strings", "on"),
              ("application_name", "turbogp_b200"), ("TimeZone", "UTC"))

    def __init__(self, executor, host: str = "127.0.0.1", port: int = 0):
        self.executor = executor
        self.sock = socket.create_server((host, port))
        self.sock.settimeout(0.2)
        self.address = self.sock.getsockname()
        self._stop = threading.Event()
        self._threads: list[threading.Thread] = []
        self._accept = threading.Thread(target=self._accept_loop, daemon=True)
        self.connections = 0

    def start(self) -> "PgWireServer":
        self._accept.start()
        return self

    def stop(self) -> None:
        self._stop.set()
        self._accept.join(timeout=5)
        self.sock.close()
        for t in self._threads:
            t.join(timeout=5)

    def _accept_loop(self) -> None:
        while not self._stop.is_set():
            try:
                conn, _ = self.sock.accept()
            except socket.timeout:
                continue
            except OSError:
                return
            self.connections += 1
            t = threading.Thread(target=self._serve, args=(conn,), daemon=True)
            self._threads.append(t)
            t.start()

    def _startup(self, conn: socket.socket) -> bool:
        while True:
            (n,) = struct.unpack("!i", _recv_exact(conn, 4))
            if not 8 <= n <= 1_000_000:
                return False
            body = _recv_exact(conn, n - 4)
            (code,) = struct.unpack("!i", body[:4])
            if code == SSL_REQUEST:
                conn.sendall(b"N")          # no TLS: the client continues in plain text
                continue
            if code == CANCEL_REQUEST:
                return False
            if code != PROTOCOL_V3:
                conn.sendall(error_response("08P01", f"unsupported protocol {code >> 16}.{code & 0xffff}"))
                return False
            out = bytearray(_msg(b"R", struct.pack("!i", 0)))
            for k, v in self.PARAMS:
                out += _msg(b"S", _cstr(k) + _cstr(v))
            out += _msg(b"K", struct.pack("!ii", os.getpid() & 0x7fffffff, id(conn) & 0x7fffffff))
            out += _msg(b"Z", b"I")
            conn.sendall(bytes(out))
            return True

    def _serve(self, conn: socket.socket) -> None:
        conn.setsockopt(socket.IPPROTO_TCP, socket.TCP_NODELAY, 1)
        try:
            if not self._startup(conn):
                return
            while not self._stop.is_set():
                kind = _recv_exact(conn, 1)
                (n,) = struct.unpack("!i", _recv_exact(conn, 4))
                if n < 4:
                    return
                body = _recv_exact(conn, n - 4)
                if kind == b"X":
                    return
                if kind == b"Q":
                    conn.sendall(self._simple_query(body.rstrip(b"\x00").decode("utf-8")))
                elif kind == b"S":
                    conn.sendall(_msg(b"Z", b"I"))
                else:
                    conn.sendall(error_response("0A000", f"unsupported message {kind!r}"))
        except (EOFError, ConnectionError, OSError):
            return
        finally:
            conn.close()

    def _simple_query(self, sql: str) -> bytes:
        out = bytearray()
        stmts = split_statements(sql)
        if not stmts:
            out += _msg(b"I")               # EmptyQueryResponse
        for s in stmts:
            try:
                names, rows = self.executor.execute(s)
                out += result_messages(names, rows)
            except SqlError as e:
                out += error_response(e.sqlstate, str(e))
                break
            except Exception as e:          # an engine failure reaches the client, not the socket
                out += error_response("XX000", f"{type(e).__name__}: {e}")
                break
        out += _msg(b"Z", b"I")
        return bytes(out)


class PgError(Exception):
    def __init__(self, sqlstate: str, message: str):
        super().__init__(f"{sqlstate}: {message}")
        self.sqlstate = sqlstate


class PgWireClient:
    """A blocking client: startup, then simple queries returning (column
    names, rows of text, command tag)."""

    def __init__(self, host: str, port: int, user: str = "turbogp", database: str = "turbogp"):
        self.sock = socket.create_connection((host, port))
        self.sock.setsockopt(socket.IPPROTO_TCP, socket.TCP_NODELAY, 1)
        params = _cstr("user") + _cstr(user) + _cstr("database") + _cstr(database) + b"\x00"
        body = struct.pack("!i", PROTOCOL_V3) + params
        self.sock.sendall(struct.pack("!i", len(body) + 4) + body)
        self.parameters: dict[str, str] = {}
        while True:
            kind, body = self._read()
            if kind == b"R" and struct.unpack("!i", body[:4])[0] != 0:
                raise PgError("28000", "authentication requested")
            if kind == b"S":
                k, v, _ = body.split(b"\x00", 2)
                self.parameters[k.decode()] = v.decode()
            if kind == b"E":
                raise PgError(*_parse_error(body))
            if kind == b"Z":
                return

    def _read(self) -> tuple[bytes, bytes]:
        kind = _recv_exact(self.sock, 1)
        (n,) = struct.unpack("!i", _recv_exact(self.sock, 4))
        return kind, _recv_exact(self.sock, n - 4)

    def query(self, sql: str):
        """Results of every statement of `sql`: [(names, rows, tag), ...];
        raises PgError on an ErrorResponse (after reading to ReadyForQuery)."""
        body = sql.encode("utf-8") + b"\x00"
        self.sock.sendall(b"Q" + struct.pack("!i", len(body) + 4) + body)
        results, names, rows, err = [], [], [], None
        while True:
            kind, body = self._read()
            if kind == b"T":
                (nf,) = struct.unpack("!h", body[:2])
                names, rows, pos = [], [], 2
                for _ in range(nf):
                    end = body.index(b"\x00", pos)
                    names.append(body[pos:end].decode())
                    pos = end + 1 + 18
            elif kind == b"D":
                (nf,) = struct.unpack("!h", body[:2])
                pos, row = 2, []
                for _ in range(nf):
                    (ln,) = struct.unpack("!i", body[pos:pos + 4])
                    pos += 4
                    row.append(None if ln < 0 else body[pos:pos + ln].decode())
                    pos += max(ln, 0)
                rows.append(tuple(row))
            elif kind == b"C":
                results.append((names, rows, body.rstrip(b"\x00").decode()))
            elif kind == b"E":
                err = _parse_error(body)
            elif kind == b"Z":
                if err:
                    raise PgError(*err)
                return results

    def close(self) -> None:
        try:
            self.sock.sendall(_msg(b"X"))
        finally:
            self.sock.close()


def _parse_error(body: bytes) -> tuple[str, str]:
    fields = {}
    for part in body.split(b"\x00"):
        if part:
            fields[chr(part[0])] = part[1:].decode()
    return fields.get("C", "XX000"), fields.get("M", "")
