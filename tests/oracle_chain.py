"""Run a golden-case chain through the oracle (one pipeline, like PipelineBuilder)."""
from oracle import oracle as O


def run_chain(img, chain, threads=1):
    if len(chain) == 1 and chain[0][0] == "resize":
        kw = chain[0][1]
        return O.resize(img, kw["hscale"], kw["vscale"], kw.get("kernel", "lanczos3"), threads=threads)
    if len(chain) == 1 and chain[0][0] == "thumbnail":
        kw = chain[0][1]
        return O.thumbnail(img, kw["target"], kw["tw"], kw["th"], kw.get("kernel", "lanczos3"),
                           kw.get("crop", False), threads=threads)
    nodes = []
    for op, kw in chain:
        if op == "reduce_h":
            nodes.append(O.make_node("reduceh", factor=kw["factor"], kernel=kw["kernel"]))
        elif op == "reduce_v":
            nodes.append(O.make_node("reducev", factor=kw["factor"], kernel=kw["kernel"]))
        elif op == "reduce":
            nodes.append(O.make_node("reduce", factor=kw["hfactor"], vfactor=kw["vfactor"], kernel=kw["kernel"]))
        elif op == "shrink_h":
            nodes.append(O.make_node("shrinkh", ufactor=kw["factor"], ceil_mode=int(kw.get("ceil", False))))
        elif op == "shrink_v":
            nodes.append(O.make_node("shrinkv", ufactor=kw["factor"], ceil_mode=int(kw.get("ceil", False))))
        else:
            raise ValueError(op)
    return O.pipeline(img, nodes, threads=threads)
