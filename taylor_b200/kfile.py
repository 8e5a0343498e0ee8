"""Reader of the LS-DYNA keyword decks MEGA takes as its model file, with
the reference's fixed-width rules (PRE_MODEL.F90:149-240,
PRE_MODEL_COUNT.f90:118-150):
  *NODE            one comment line, then records (I8, 3F16.0, 2I8): id, x, y, z
  *ELEMENT_SOLID   records (10I8): id, part, eight node ids; every card
                   starts an element block; a block is tetrahedral (type 1)
                   when its last element repeats its seventh node as its
                   eighth, hexahedral (type 2) otherwise
  *SET_NODE_LIST   the set id, then records (8I10) of node ids (zeros end a
                   record)
Lines starting with '$' are comments.  The arrays come back ready for
mega_pre_model (connectivity 0-based here, the element types per element).
"""
import numpy as np


def _is_card(line):
    return line.startswith("*")


def read_k(path_or_text):
    """dict(coo (n, 3) by node id, elems (E, 8) 0-based, block (E),
    block_type (nblocks), eltype (E), sets {id: 1-based node ids})."""
    text = path_or_text
    if "\n" not in path_or_text:
        with open(path_or_text) as f:
            text = f.read()
    lines = text.splitlines()
    nodes, elems, blocks, sets = {}, [], [], {}
    i, nblock = 0, 0
    while i < len(lines):
        card = lines[i].strip()
        if card == "*NODE":
            i += 2  # the comment line after the card is skipped unread
            while i < len(lines) and not _is_card(lines[i]):
                ln = lines[i]
                if ln.strip() and not ln.startswith("$"):
                    nodes[int(ln[0:8])] = (float(ln[8:24]), float(ln[24:40]), float(ln[40:56]))
                i += 1
            continue
        if card == "*ELEMENT_SOLID":
            nblock += 1
            i += 1
            while i < len(lines) and not _is_card(lines[i]):
                ln = lines[i]
                if ln.strip() and not ln.startswith("$"):
                    elems.append([int(ln[8 * k:8 * k + 8]) for k in range(2, 10)])
                    blocks.append(nblock - 1)
                i += 1
            continue
        if card == "*SET_NODE_LIST":
            sid = int(lines[i + 1].split()[0])
            i += 2
            ids = []
            while i < len(lines) and not _is_card(lines[i]):
                ln = lines[i]
                if not ln.startswith("$"):
                    for k in range(8):
                        f = ln[10 * k:10 * k + 10].strip()
                        if f and int(f) != 0:
                            ids.append(int(f))
                i += 1
            sets[sid] = np.array(ids, np.int32)
            continue
        i += 1
    n = max(nodes) if nodes else 0
    coo = np.zeros((n, 3))
    for k, v in nodes.items():
        coo[k - 1] = v
    el = np.array(elems, np.int32).reshape(-1, 8)
    block = np.array(blocks, np.int32)
    btype = np.full(nblock, 2, np.int32)
    for b in range(nblock):
        last = np.flatnonzero(block == b)
        if len(last) and el[last[-1], 6] == el[last[-1], 7]:
            btype[b] = 1
    return dict(coo=coo, elems=el - 1, block=block, block_type=btype, eltype=btype[block] if len(block) else block,
                sets=sets)
