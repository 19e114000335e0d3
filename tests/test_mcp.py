"""The MCP server's protocol on the CPU (shaderous_b200/mcp.py, after tools/headless/mcp.mjs):
JSON-RPC 2.0 lines over stdio, initialize / ping / tools/list / tools/call, notifications without
an answer, parse and method errors, and tools that need no GPU (describe, check_setup, errors);
a tool that fails answers with isError and its message."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def converse(msgs, extra_lines=()):
    text = "\n".join(json.dumps(m) for m in msgs) + "\n" + "\n".join(extra_lines) + "\n"
    p = subprocess.run([sys.executable, "-m", "shaderous_b200.mcp"], input=text, capture_output=True, text=True,
                       cwd=ROOT, timeout=300)
    assert p.returncode == 0, p.stderr
    return [json.loads(line) for line in p.stdout.splitlines()]


def body(reply):
    return json.loads(reply["result"]["content"][0]["text"])


def test_protocol_and_cpu_tools():
    out = converse([
        {"jsonrpc": "2.0", "id": 1, "method": "initialize", "params": {"protocolVersion": "2025-06-18"}},
        {"jsonrpc": "2.0", "method": "notifications/initialized"},
        {"jsonrpc": "2.0", "id": 2, "method": "ping"},
        {"jsonrpc": "2.0", "id": 3, "method": "tools/list"},
        {"jsonrpc": "2.0", "id": 4, "method": "tools/call", "params": {"name": "describe", "arguments": {}}},
        {"jsonrpc": "2.0", "id": 5, "method": "tools/call",
         "params": {"name": "describe", "arguments": {"problem": "kh"}}},
        {"jsonrpc": "2.0", "id": 6, "method": "tools/call",
         "params": {"name": "check_setup", "arguments": {"setup": "problem=sedov&dim=3&n=64&amr=3"}}},
        {"jsonrpc": "2.0", "id": 7, "method": "tools/call",
         "params": {"name": "check_setup", "arguments": {"setup": "problem=nope"}}},
        {"jsonrpc": "2.0", "id": 8, "method": "tools/call", "params": {"name": "run", "arguments": {"steps": 3}}},
        {"jsonrpc": "2.0", "id": 9, "method": "tools/call", "params": {"name": "screenshot", "arguments": {}}},
        {"jsonrpc": "2.0", "id": 10, "method": "tools/call", "params": {"name": "errors", "arguments": {}}},
        {"jsonrpc": "2.0", "id": 11, "method": "resources/list"},
    ], extra_lines=["{not json"])
    by = {r["id"]: r for r in out}
    assert len(out) == 12  # eleven answers (the notification has none) and the parse error
    assert by[1]["result"]["serverInfo"]["name"] == "shaderous-b200"
    assert by[1]["result"]["capabilities"] == {"tools": {}}
    assert by[2]["result"] == {}
    names = {t["name"] for t in by[3]["result"]["tools"]}
    assert {"describe", "load", "run", "diagnostics", "slice", "probe", "save_athdf", "load_athdf"} <= names
    assert all(t["inputSchema"]["type"] == "object" for t in by[3]["result"]["tools"])
    assert {p["id"] for p in body(by[4])["problems"]} >= {"sod", "kelvin-helmholtz", "sedov", "taylor-green"}
    assert body(by[5])["id"] == "kelvin-helmholtz"
    chk = body(by[6])
    assert chk["grid"] == "adaptive" and chk["setup"]["amr"] == 3
    assert by[7]["result"]["isError"] and "unknown problem" in by[7]["result"]["content"][0]["text"]
    assert by[8]["result"]["isError"] and "load first" in by[8]["result"]["content"][0]["text"]
    assert by[9]["error"]["code"] == -32602  # not a tool this server has
    errs = body(by[10])["errors"]
    assert len(errs) == 2 and errs[0].startswith("run:")
    assert by[11]["error"]["code"] == -32601
    assert by[None]["error"]["code"] == -32700
