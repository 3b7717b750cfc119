"""Query execution with the reference's frontend surface
(system/tmine/frontend.py:38-159): ``HeavyRes`` loads the graph once,
``Mining.run(yaml)`` runs one query, ``MiningSingle(yaml).run()`` both.

Differences by design: no per-query code generation or nvcc (one prebuilt
plugin serves every motif), the device graph stays resident across queries
of the same graph (the reference re-uploads it per query), and one GPU only.
"""
from timeit import default_timer as timer

import numpy as np

from . import core, locations, utils
from .Query import Query


class HeavyRes:
    def __init__(self, graph: str, gpu: int):
        if int(gpu) > 1:
            raise NotImplementedError("multi-GPU execution is not on this path (one GPU only)")
        self.graph = graph
        self.gpu = int(gpu)
        self.eloader = core.data.EdgeListLoader(graph)
        self.floader = core.data.FeatureLoader(self.eloader, locations.randFilePath())
        self.gloader = core.data.GraphDataLoader(self.eloader, self.floader)
        self.hostGraph = self.gloader.createGraphData()


class Mining:
    def __init__(self, pathToGraph: str, gpu: int):
        self.heavy = HeavyRes(pathToGraph, gpu)
        self.libManager = core.GPUWorkerLibManager()
        self.dataManager = core.data.MakeGraphDataManager(max(1, int(gpu)))
        self.libName = None
        self.exec = None

    def makePlugin(self, query: Query):
        """Open the prebuilt plugin (the reference generates and compiles one
        per query here)."""
        if self.libName is None:
            path = locations.dynLibPath()
            self.libManager.openLib(path)
            self.libName = utils.libFileToLibName(path)

    def _execution(self):
        if self.exec is None:
            self.exec = core.SingleGPUExecution(self.dataManager, 0)
            self.exec.setHostGraph(self.heavy.hostGraph)  # resident for every later query
        return self.exec

    def processSingle(self, query: Query, out=print):
        hostMotif = core.data.HostMotifData(query.pattern())
        w = self.libManager.construct(self.libName, 0)
        opts = query.options()
        w.configure(opts.enumNum() if opts.enumerate() else 0, opts.flags())
        mu, mv = hostMotif.motifEdges()
        cons = query.constraints().compile(mu, mv)
        w.setConstraints(None if cons.empty else bytes(cons.to_struct()))
        ex = self._execution()
        ex.setHostMotif(hostMotif)
        ex.setWorker(w)
        start = timer()
        ex.run(query.constraints().delta())
        end = timer()
        cn, tm = w.count(), w.time()
        out("@@@ [output starts]", flush=True)
        rows = None
        if not opts.enumerate():
            out(f"{cn}, {tm}, {end - start}")
        else:
            rows = np.array(w.printEnum(opts.enumNum()), dtype=np.int64).reshape(-1, hostMotif.numEdges)
            for r in rows:
                out(" ".join(map(str, r)))
        out("@@@ [output ends]")
        del w
        return (cn, tm, end - start) if rows is None else (cn, tm, end - start, rows)

    def processQuery(self, query: Query, out=print):
        if query.options().gpu() != self.heavy.gpu:
            raise ValueError(f"query asks for {query.options().gpu()} GPUs, loaded for {self.heavy.gpu}")
        import os
        if os.path.abspath(query.graph()) != os.path.abspath(self.heavy.graph):
            raise ValueError(f"cannot process query {query.name}: graph {query.graph()} is not loaded")
        self.makePlugin(query)
        return self.processSingle(query, out)

    def run(self, pathToQuery: str, out=print):
        return self.processQuery(Query(pathToQuery), out)


class MiningSingle(Mining):
    def __init__(self, pathToQuery: str):
        query = Query(pathToQuery)
        super().__init__(query.graph(), query.options().gpu())
        self.query = query

    def run(self, out=print):
        return self.processQuery(self.query, out)
