"""Oracle for unstructured grids (test infrastructure only).

Restates, in plain Python and numpy:
  * unstructured::domain_descriptor (unstructured/user_concepts.hpp:37-175) and make_outer_lids
    (:88-113): repeated halo gids take their local ids in ascending order (the reference uses
    std::unordered_multimap's equal_range order; every local id of one gid receives the value of
    the same owner, so the exchanged values do not depend on it);
  * halo_generator (:180-256), all outer gids or an explicit list;
  * make_pattern_impl<unstructured grid>::apply without domain hints (unstructured/pattern.hpp:
    187-370): the send list of owner i towards domain o is the subsequence of o's halo gids that are
    inner to i (in o's halo order), the receive list its local ids in o; tags
    (i << num_bits(#domains)) | id(o), maps ordered by tag;
  * the exchange (data_descriptor get/set, user_concepts.hpp:383-452, with the message buffer
    removed) and its adjoint in receive-map order, column by column;
  * make_pattern with a receive domain ids generator (unstructured/pattern.hpp:371-588);
  * the in-place receive (unstructured/communication_object_ipr.hpp:105-186): a neighbour's
    message lands on consecutive rows from the first index of its receive list.

Fields are numpy arrays of shape (n,) or (n, levels) — either memory order.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


class Domain:
    def __init__(self, id_: int, gids, outer_lids):
        self.id = int(id_)
        self.gids = [int(g) for g in gids]
        self.outer_lids = [int(x) for x in outer_lids]
        outer = set(self.outer_lids)
        if len(outer) != len(self.outer_lids):
            raise ValueError("repeated outer (local) index")
        self.inner: dict[int, int] = {}
        self.outer: dict[int, list[int]] = {}
        self.outer_gids: list[int] = []
        for lid, g in enumerate(self.gids):
            if lid in outer:
                self.outer.setdefault(g, []).append(lid)
                self.outer_gids.append(g)
            else:
                if g in self.inner:
                    raise ValueError("repeated inner (global) index")
                self.inner[g] = lid

    def make_outer_lids(self, gids):
        lids, used = [], {}
        for g in gids:
            if g not in self.outer:
                continue
            k = used.get(g, 0)
            if k >= len(self.outer[g]):
                raise ValueError("halo gid does not have an associated lid in the domain")
            lids.append(self.outer[g][k])
            used[g] = k + 1
        for g, k in used.items():
            if k != len(self.outer[g]):
                raise ValueError("halo gid occurs not often enough")
        return lids


@dataclass
class Entry:
    neighbor: int
    tag: int
    lids: list = field(default_factory=list)


def _num_bits(n: int) -> int:
    return 1 if n == 0 else 1 + _num_bits(n >> 1)


def make_pattern(domains: list[Domain], halo_gids=None):
    """Receive and send entries per domain. halo_gids: None (all outer gids) or one gid list per
    domain."""
    n = len(domains)
    halos = []
    for i, d in enumerate(domains):
        lids = d.make_outer_lids(d.outer_gids if halo_gids is None else halo_gids[i])
        halos.append([d.gids[l] for l in lids])
    shift = _num_bits(n)
    recv = [dict() for _ in range(n)]
    send = [dict() for _ in range(n)]
    for o in range(n):
        for i in range(n):
            tag = (i << shift) | domains[o].id
            s = [domains[i].inner[g] for g in halos[o] if g in domains[i].inner]
            if not s:
                continue
            g_list = [g for g in halos[o] if g in domains[i].inner]
            send[i][tag] = Entry(o, tag, s)
            recv[o][tag] = Entry(i, tag, domains[o].make_outer_lids(g_list))
    max_tag = (n << shift) | max(d.id for d in domains)
    return ([[recv[d][t] for t in sorted(recv[d])] for d in range(n)],
            [[send[d][t] for t in sorted(send[d])] for d in range(n)], max_tag)


def make_pattern_hinted(domains: list[Domain], hints, halo_gids=None):
    """make_pattern with a receive domain ids generator (unstructured/pattern.hpp:371-588), one
    process. hints[i] = (owner ids, remote indices) per halo element of domain i in the halo
    generator's order. Receive entries group the halo elements by owner (ascending owner id),
    the owner's send entry lists the remote indices in the receiver's order; tag (owner id << 7) +
    receiver id; maximum tag (max id << 7) + max id. A remote index must be an inner element."""
    n = len(domains)
    idx = {d.id: i for i, d in enumerate(domains)}
    recv = [dict() for _ in range(n)]
    send = [dict() for _ in range(n)]
    for i, d in enumerate(domains):
        lids = d.make_outer_lids(d.outer_gids if halo_gids is None else halo_gids[i])
        owners, remote = hints[i]
        if len(owners) != len(lids) or len(remote) != len(lids):
            raise ValueError("one receive domain id and remote index per halo element")
        for lid, o, r in zip(lids, owners, remote):
            od = domains[idx[o]]
            if not (0 <= r < len(od.gids)) or r in set(od.outer_lids):
                raise ValueError(f"remote index {r} of domain {o} is not an inner element")
            tag = ((o << 7) + d.id) & 0xFFFFFFFF
            recv[i].setdefault(o, Entry(idx[o], tag)).lids.append(lid)
            send[idx[o]].setdefault(d.id, Entry(i, tag)).lids.append(r)
    m = max(d.id for d in domains)
    return ([[recv[i][k] for k in sorted(recv[i])] for i in range(n)],
            [[send[i][k] for k in sorted(send[i])] for i in range(n)], (m << 7) + m)


def _pairs(recv, send):
    """(receiver, sender, receive lids, send lids) in receive-map order."""
    for d, entries in enumerate(recv):
        for en in entries:
            s = next(x for x in send[en.neighbor] if x.neighbor == d and x.tag == en.tag)
            yield d, en.neighbor, np.asarray(en.lids), np.asarray(s.lids)


def exchange(recv, send, fields) -> None:
    for d, e, R, S in _pairs(recv, send):
        fields[d][R] = fields[e][S]


def adjoint(recv, send, grads) -> None:
    """owner += halo in receive-map order, then halo = 0 (np.add.at adds repeated owners in order)."""
    for d, e, R, S in _pairs(recv, send):
        h = grads[d][R].copy()
        if grads[e].ndim == 1:
            np.add.at(grads[e], S, h)
        else:
            np.add.at(grads[e], (S, slice(None)), h)
        grads[d][R] = 0


def in_place_rows(recv, domains):
    """Rows written by GHEX's in-place receive (unstructured/communication_object_ipr.hpp:127-141):
    a neighbour's message is received as raw bytes at the address of the first index of its
    receive list, so its k-th value lands on row first + k. Raises ValueError where those rows
    are not halo rows of the domain received once (the outcome would depend on copy order)."""
    out = []
    for d, entries in enumerate(recv):
        outer = set(domains[d].outer_lids)
        claimed = set()
        rows = []
        for en in entries:
            r = list(range(en.lids[0], en.lids[0] + len(en.lids)))
            for x in r:
                if x not in outer or x in claimed:
                    raise ValueError(f"in-place receive: the halo of domain {domains[d].id} received from domain "
                                     f"{domains[en.neighbor].id} is not stored on consecutive halo rows")
                claimed.add(x)
            rows.append(r)
        out.append(rows)
    return out


def exchange_in_place(recv, send, fields, domains) -> None:
    """The in-place receive exchange of one field per domain: the sender packs its values in the
    receiver's order, levels innermost (data_descriptor::get, user_concepts.hpp:415-440), the
    receiver stores them on in_place_rows."""
    rows = in_place_rows(recv, domains)
    for d, entries in enumerate(recv):
        for en, r in zip(entries, rows[d]):
            s = next(x for x in send[en.neighbor] if x.neighbor == d and x.tag == en.tag)
            fields[d][np.asarray(r)] = fields[en.neighbor][np.asarray(s.lids)]
