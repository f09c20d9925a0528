"""One process's block of subdomains of the numpy oracle, with the operators the partitioned driver
(espreso_b200.partitioned) asks of a block.  Test infrastructure: the gloo tests run the driver's
collectives between CPU processes on these blocks; on a GPU the product's blocks are FETI4I instances."""
import numpy as np


class OracleBlock:
    def __init__(self, OP, first, count, P):
        self.OP = OP
        self.first, self.count = first, count
        self.sub = OP.sub[first:first + count]
        self.n_lambda = OP.n_lambda
        self.P = P
        num = OP.num
        self.mult = np.zeros(P.n_nodes)
        for nodes in num.dom_nodes:
            self.mult[nodes] += 1

    def coarse_blocks(self):
        return [(self.first + k, s.lam.astype(np.int64), s.G) for k, s in enumerate(self.sub)]

    def dual_rhs(self):
        b = np.zeros(self.n_lambda)
        eb = {}
        for k, s in enumerate(self.sub):
            kf = s.kplus(s.f)
            np.add.at(b, s.lam, s.sign * kf[s.dof] - s.c)
            eb[self.first + k] = -(s.R.T @ s.f)
        return b, eb

    def apply_F(self, x, y):
        xv, yv = x.numpy(), y.numpy()
        for s in self.sub:
            np.add.at(yv, s.lam, s.S @ xv[s.lam])

    def precondition(self, x, y):
        from oracle import feti as OF
        xv, yv = x.numpy(), y.numpy()
        for s in self.sub:
            xi = xv[s.lam] * s.w
            if self.prec in (OF.PREC_LUMPED, OF.PREC_MAGIC):
                u = np.zeros(s.K.shape[0])
                np.add.at(u, s.dof, s.sign * xi)
                yi = s.sign * (s.K @ u)[s.dof]
            elif self.prec == OF.PREC_WEIGHT:
                yi = xi
            else:
                u = np.zeros(s.tdofs.size)
                np.add.at(u, s.trow, s.sign * xi)
                M = s.Sdir if self.prec == OF.PREC_DIRICHLET else s.Ssd
                yi = s.sign * (M @ u)[s.trow]
            np.add.at(yv, s.lam, yi * s.w)

    def primal(self, lam, alpha_blocks):
        dpn = self.OP.num.dpn
        acc = np.zeros((self.P.n_nodes, dpn))
        for k, s in enumerate(self.sub):
            d = self.first + k
            g = s.f.copy()
            np.add.at(g, s.dof, -s.sign * lam[s.lam])
            u = s.kplus(g) + s.R @ alpha_blocks[d]
            nodes = self.OP.num.dom_nodes[d]
            acc[nodes] += u.reshape(-1, dpn) / self.mult[nodes, None]
        return acc.ravel()
