// mesh.cpp -- reliability-guided mesh solve on top of the batched GPU solve.
//
// Reference: Mesh::solve_impl (src/mesh.rs:628-764), solve_node
// (:1068-1106), solve_neighbours_from (:1112-1154), expand_parallel
// (:1169-1252), greedy_graph_colour (:1884-1903), Adjacency / connectivity
// (:1699-1872), find_seed_node (:1682-1697), precondition_warp /
// affine_field_fit / ols_solve / project_warp (:2101-2233), store_result
// (:2385-2402).  The propagation order, the trusted sets, the two attempts of
// solve_node and the fold order follow the reference exactly; what changes is
// that every graph colour of a layer-RG round (a set of subsets with no
// shared mesh edge, solved independently in the reference by rayon) is one
// batch, and the zero-warp second attempts of that colour a second batch.
// The serial RG cascade issues one batch per node.  The driver is written
// against a batch-solver callback: gpv_mesh_solve plugs in the GPU solve,
// and any other solver (a CPU one, to check the driver) can be plugged into
// gpv_mesh_drive.  Corrections (:1265-1414), element strains and the
// compatibility check are host post-processing left to the caller.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <queue>
#include <set>
#include <vector>

#include "internal.h"

namespace gpv {
namespace {

struct Adjacency {
    std::vector<std::vector<int64_t>> full, edge;
};

// connectivity (src/mesh.rs:1705-1772): full = every other node of every
// element containing idx; edge (order-2 meshes) = midpoint <-> corner sides.
Adjacency build_adjacency(const int64_t *el, int64_t n_el, int npe, int64_t n_nodes) {
    Adjacency A;
    A.full.assign(n_nodes, {});
    A.edge.assign(n_nodes, {});
    std::vector<std::set<int64_t>> full(n_nodes), edge(n_nodes);
    static const int sides[6][2] = {{3, 5}, {3, 4}, {4, 5}, {0, 1}, {1, 2}, {0, 2}};
    for (int64_t e = 0; e < n_el; e++) {
        const int64_t *row = el + e * npe;
        for (int k = 0; k < npe; k++) {
            const int64_t idx = row[k];
            for (int j = 0; j < npe; j++)
                if (row[j] != idx) full[idx].insert(row[j]);
            if (npe == 6)
                for (int j = 0; j < 2; j++)
                    if (row[sides[k][j]] != idx) edge[idx].insert(row[sides[k][j]]);
        }
    }
    for (int64_t i = 0; i < n_nodes; i++) {
        A.full[i].assign(full[i].begin(), full[i].end());
        if (npe == 6) A.edge[i].assign(edge[i].begin(), edge[i].end());
        else A.edge[i] = A.full[i];
    }
    return A;
}

// Inverse of the OLS normal-equation matrix, computed the way the
// reference's linear-algebra crate (nalgebra, DMatrix::try_inverse) does:
// 3x3 by cofactors (an exactly-zero determinant = singular), larger by LU
// with partial pivoting (an exactly-zero pivot = singular).
bool try_inverse(std::vector<double> a, int m, std::vector<double> &inv) {
    inv.assign(m * m, 0.0);
    if (m == 3) {
        const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
        const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
        if (det == 0.0) return false;
        inv[0] = c00 / det;
        inv[1] = (a[2] * a[7] - a[1] * a[8]) / det;
        inv[2] = (a[1] * a[5] - a[2] * a[4]) / det;
        inv[3] = c01 / det;
        inv[4] = (a[0] * a[8] - a[2] * a[6]) / det;
        inv[5] = (a[2] * a[3] - a[0] * a[5]) / det;
        inv[6] = c02 / det;
        inv[7] = (a[1] * a[6] - a[0] * a[7]) / det;
        inv[8] = (a[0] * a[4] - a[1] * a[3]) / det;
        return true;
    }
    // LU with partial pivoting (multipliers kept below the diagonal), then
    // per column of the identity: permute, unit-lower solve, upper solve,
    // both column-oriented.
    std::vector<int> perm(m);
    for (int i = 0; i < m; i++) perm[i] = i;
    for (int k = 0; k < m; k++) {
        int piv = k;
        for (int i = k + 1; i < m; i++)
            if (std::fabs(a[i * m + k]) > std::fabs(a[piv * m + k])) piv = i;
        if (a[piv * m + k] == 0.0) return false;
        if (piv != k) {
            for (int j = 0; j < m; j++) std::swap(a[k * m + j], a[piv * m + j]);
            std::swap(perm[k], perm[piv]);
        }
        for (int i = k + 1; i < m; i++) {
            a[i * m + k] /= a[k * m + k];
            const double f = a[i * m + k];
            for (int j = k + 1; j < m; j++) a[i * m + j] -= f * a[k * m + j];
        }
    }
    std::vector<double> b(m);
    for (int c = 0; c < m; c++) {
        for (int r = 0; r < m; r++) b[r] = perm[r] == c ? 1.0 : 0.0;
        for (int k = 0; k < m; k++)
            for (int r = k + 1; r < m; r++) b[r] -= a[r * m + k] * b[k];
        for (int k = m - 1; k >= 0; k--) {
            b[k] /= a[k * m + k];
            for (int r = 0; r < k; r++) b[r] -= a[r * m + k] * b[k];
        }
        for (int r = 0; r < m; r++) inv[r * m + c] = b[r];
    }
    return true;
}

struct MeshRun {
    gpv_batch_solver_fn solver;
    void *solver_user;
    const double *nodes;
    int64_t n;
    const gpv_mesh_params *mp;
    int p_len;
    std::vector<char> stored, propagated, quality_ok;
    std::vector<double> c_zncc;   // max(c_zncc, 0), as stored by store_result
    std::vector<double> p;        // n x 12
    gpv_subset_result *out;
    int32_t *rounds;
    int64_t done = 0, batches = 0, solves = 0, retries = 0;
    int round = 0;
    // max-heap of (c_zncc bits, node) (src/mesh.rs:649)
    std::priority_queue<std::pair<uint64_t, int64_t>> queue;

    double px(int64_t i) const { return nodes[2 * i]; }
    double py(int64_t i) const { return nodes[2 * i + 1]; }

    // ols_solve (src/mesh.rs:2220-2233): (A^T A)^-1 A^T y
    bool ols(const std::vector<std::vector<double>> &rows, const std::vector<double> &y, std::vector<double> &x) const {
        const int m = (int)rows[0].size();
        std::vector<double> ata(m * m, 0.0), aty(m, 0.0), inv;
        for (size_t r = 0; r < rows.size(); r++)
            for (int i = 0; i < m; i++) {
                aty[i] += rows[r][i] * y[r];
                for (int j = 0; j < m; j++) ata[i * m + j] += rows[r][i] * rows[r][j];
            }
        if (!try_inverse(ata, m, inv)) return false;
        x.assign(m, 0.0);
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) x[i] += inv[i * m + j] * aty[j];
        return true;
    }

    // precondition_warp (src/mesh.rs:2130-2151)
    void precondition(int64_t target, const std::vector<int64_t> &trusted, double *w) const {
        for (int k = 0; k < 12; k++) w[k] = 0.0;
        const double tx = px(target), ty = py(target);
        if (trusted.size() >= 3) {  // affine_field_fit (:2170-2215)
            const bool quad = p_len >= 12 && trusted.size() >= 6;
            std::vector<std::vector<double>> rows;
            std::vector<double> u, v, cu, cv;
            for (int64_t i : trusted) {
                const double dx = px(i) - tx, dy = py(i) - ty;
                if (quad) rows.push_back({1.0, dx, dy, dx * dx, dx * dy, dy * dy});
                else rows.push_back({1.0, dx, dy});
                u.push_back(p[12 * i + 0]);
                v.push_back(p[12 * i + 1]);
            }
            if (ols(rows, u, cu) && ols(rows, v, cv)) {
                w[0] = cu[0]; w[1] = cv[0]; w[2] = cu[1]; w[3] = cv[1]; w[4] = cu[2]; w[5] = cv[2];
                if (quad) {
                    w[6] = 2.0 * cu[3]; w[7] = 2.0 * cv[3]; w[8] = cu[4];
                    w[9] = cv[4]; w[10] = 2.0 * cu[5]; w[11] = 2.0 * cv[5];
                }
                return;
            }
        }
        if (!trusted.empty()) {  // Taylor projection from the best neighbour (:2141-2148)
            int64_t best = trusted[0];
            for (int64_t i : trusted)
                if (c_zncc[i] >= c_zncc[best]) best = i;  // Iterator::max_by keeps the last maximum
            const double dx = tx - px(best), dy = ty - py(best);
            const double *q = &p[12 * best];
            for (int k = 0; k < p_len; k++) w[k] = q[k];
            if (p_len >= 6) {  // project_warp (:2107-2122)
                w[0] = q[0] + q[2] * dx + q[4] * dy;
                w[1] = q[1] + q[3] * dx + q[5] * dy;
            }
            if (p_len >= 12) {
                w[0] += 0.5 * q[6] * dx * dx + q[8] * dx * dy + 0.5 * q[10] * dy * dy;
                w[1] += 0.5 * q[7] * dx * dx + q[9] * dx * dy + 0.5 * q[11] * dy * dy;
                w[2] = q[2] + q[6] * dx + q[8] * dy;
                w[3] = q[3] + q[7] * dx + q[9] * dy;
                w[4] = q[4] + q[8] * dx + q[10] * dy;
                w[5] = q[5] + q[9] * dx + q[11] * dy;
            }
        }
    }

    // One solver call.  Subsets that Subset::new rejects (src/subset.rs:
    // 853-892, an Err that aborts Mesh::solve) or that hit the reference's
    // singular-matrix panics (:1143, :520, :595) end the mesh solve with an
    // error naming the node.
    int solve(const std::vector<int64_t> &ids, std::vector<gpv_subset_desc> &d, std::vector<gpv_subset_result> &r,
              double tolerance) {
        r.assign(d.size(), gpv_subset_result{});
        batches++;
        solves += (int64_t)d.size();
        if (int rc = solver(solver_user, d.data(), (int64_t)d.size(), tolerance, r.data())) return rc;
        for (size_t k = 0; k < r.size(); k++) {
            const int st = r[k].status;
            if (st == GPV_EMPTY_MASK || st == GPV_FEATURELESS || st == GPV_SINGULAR_H || st == GPV_SINGULAR_WDELTA ||
                st == GPV_INVALID_SUBSET || st == GPV_TIMEOUT || st == GPV_CANCELLED) {
                static const char *what[] = {"ok", "empty subset mask", "featureless subset", "singular Hessian",
                                             "singular warp increment", "non-finite", "timed out", "cancelled",
                                             "invalid subset"};
                set_error("mesh node " + std::to_string(ids[k]) + ": " + what[st]);
                return GPV_ERR_INVALID;
            }
        }
        return GPV_SUCCESS;
    }

    // solve_node for a set of nodes at once (src/mesh.rs:1068-1106): attempt
    // A with its preconditioned (or forced) warp; attempt B with the zero warp
    // for nodes whose A is not quality_ok and whose A warp was not already zero.
    int solve_nodes(const std::vector<int64_t> &ids, const std::vector<std::vector<double>> &p0, double tolerance,
                    std::vector<gpv_subset_result> &res) {
        std::vector<gpv_subset_desc> d(ids.size());
        for (size_t k = 0; k < ids.size(); k++) {
            std::memset(&d[k], 0, sizeof(d[k]));
            d[k].coord[0] = px(ids[k]);
            d[k].coord[1] = py(ids[k]);
            d[k].order = mp->subset_order;
            d[k].radius = mp->radius;
            for (int j = 0; j < p_len; j++) d[k].p0[j] = p0[k][j];
        }
        std::vector<gpv_subset_result> ra;
        if (int rc = solve(ids, d, ra, tolerance)) return rc;
        std::vector<size_t> retry;
        for (size_t k = 0; k < ids.size(); k++) {
            if (ra[k].quality_ok) continue;
            bool zero = true;
            for (int j = 0; j < p_len; j++) zero = zero && p0[k][j] == 0.0;
            if (!zero) retry.push_back(k);
        }
        res = ra;
        if (!retry.empty()) {
            std::vector<gpv_subset_desc> db;
            std::vector<int64_t> idb;
            for (size_t k : retry) {
                gpv_subset_desc z = d[k];
                for (int j = 0; j < 12; j++) z.p0[j] = 0.0;
                db.push_back(z);
                idb.push_back(ids[k]);
            }
            retries += (int64_t)retry.size();
            std::vector<gpv_subset_result> rb;
            if (int rc = solve(idb, db, rb, tolerance)) return rc;
            for (size_t t = 0; t < retry.size(); t++) {
                const size_t k = retry[t];
                if (rb[t].quality_ok || rb[t].c_zncc > ra[k].c_zncc) res[k] = rb[t];
            }
        }
        return GPV_SUCCESS;
    }

    // store_result (src/mesh.rs:2385-2402) + progress::node_done (src/progress.rs:35-38)
    int store(int64_t idx, const gpv_subset_result &r) {
        quality_ok[idx] = r.quality_ok != 0;
        c_zncc[idx] = std::fmax(r.c_zncc, 0.0);  // f64::max: a NaN gives 0
        for (int k = 0; k < 12; k++) p[12 * idx + k] = k < p_len ? r.p[k] : 0.0;
        out[idx] = r;
        if (rounds) rounds[idx] = round;
        stored[idx] = 1;
        done++;
        if (mp->progress && mp->progress(mp->progress_user, done, n)) {
            set_error("solve cancelled");
            return GPV_ERR_CANCELLED;
        }
        return GPV_SUCCESS;
    }

    void push(int64_t idx) {
        uint64_t bits;
        std::memcpy(&bits, &c_zncc[idx], sizeof bits);
        queue.push({bits, idx});
    }

    std::vector<int64_t> trusted_of(const Adjacency &adj, int64_t nb) const {
        std::vector<int64_t> t;
        for (int64_t x : adj.full[nb])
            if (stored[x] && quality_ok[x]) t.push_back(x);
        return t;
    }

    // expand_parallel (src/mesh.rs:1169-1252)
    int expand(const Adjacency &adj, const std::vector<int64_t> &roots) {
        std::vector<int64_t> cand;
        for (int64_t r : roots)
            for (int64_t nb : adj.edge[r])
                if (!stored[nb]) cand.push_back(nb);
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        if (cand.empty()) return GPV_SUCCESS;
        // greedy_graph_colour (:1884-1903) over the full adjacency
        std::vector<int64_t> colour(cand.size(), -1);
        int64_t n_col = 0;
        for (size_t i = 0; i < cand.size(); i++) {
            std::vector<char> used;
            for (int64_t nb : adj.full[cand[i]]) {
                auto it = std::lower_bound(cand.begin(), cand.end(), nb);
                if (it != cand.end() && *it == nb) {
                    const int64_t cn = colour[it - cand.begin()];
                    if (cn >= 0) {
                        if ((int64_t)used.size() <= cn) used.resize(cn + 1, 0);
                        used[cn] = 1;
                    }
                }
            }
            int64_t k = 0;
            while (k < (int64_t)used.size() && used[k]) k++;
            colour[i] = k;
            n_col = std::max(n_col, k + 1);
        }
        for (int64_t c = 0; c < n_col; c++) {
            std::vector<int64_t> ids;
            std::vector<std::vector<double>> p0;
            for (size_t i = 0; i < cand.size(); i++) {
                if (colour[i] != c) continue;
                ids.push_back(cand[i]);
                std::vector<double> w(12);
                precondition(cand[i], trusted_of(adj, cand[i]), w.data());
                p0.push_back(w);
            }
            std::vector<gpv_subset_result> res;
            if (int rc = solve_nodes(ids, p0, mp->tolerance, res)) return rc;
            for (size_t k = 0; k < ids.size(); k++) {  // ascending node order (ids are sorted)
                if (int rc = store(ids[k], res[k])) return rc;
                push(ids[k]);
            }
            round++;
        }
        return GPV_SUCCESS;
    }

    // solve_neighbours_from (src/mesh.rs:1112-1154), one node per batch
    int neighbours_from(const Adjacency &adj, int64_t cur) {
        for (int64_t nb : adj.edge[cur]) {
            if (stored[nb]) continue;
            std::vector<double> w(12);
            precondition(nb, trusted_of(adj, nb), w.data());
            std::vector<gpv_subset_result> res;
            if (int rc = solve_nodes({nb}, {w}, mp->tolerance, res)) return rc;
            if (int rc = store(nb, res[0])) return rc;
            push(nb);
            round++;
        }
        return GPV_SUCCESS;
    }
};

}  // namespace

int mesh_drive(const double *nodes, int64_t n_nodes, const int64_t *elements, int64_t n_elements,
               int32_t nodes_per_element, const gpv_mesh_params *mp, gpv_batch_solver_fn solver, void *solver_user,
               gpv_subset_result *out, int32_t *rounds, gpv_mesh_stats *stats) {
    if (!nodes || !elements || !mp || !solver || !out || n_nodes < 1 || n_elements < 1 ||
        (nodes_per_element != 3 && nodes_per_element != 6)) {
        set_error("invalid mesh arguments");
        return GPV_ERR_INVALID;
    }
    if (mp->subset_order < 1 || mp->subset_order > 2 || mp->radius < 1) {
        set_error("mesh solves use subset_order 1 or 2 and radius >= 1");
        return GPV_ERR_INVALID;
    }
    if (mp->texture != 0 && mp->texture != 1) {
        set_error("texture must be 0 (deformable) or 1 (rigid)");
        return GPV_ERR_INVALID;
    }
    if (mp->method != 0 && mp->method != 1) {
        set_error("method must be 0 (ICGN) or 1 (FAGN)");
        return GPV_ERR_INVALID;
    }
    if (mp->layer_rg && (mp->batch_factor < 1 || mp->max_workers < 1)) {
        set_error("layer-RG needs batch_factor >= 1 and max_workers >= 1");
        return GPV_ERR_INVALID;
    }
    for (int64_t i = 0; i < n_elements * nodes_per_element; i++)
        if (elements[i] < 0 || elements[i] >= n_nodes) {
            set_error("element references a node outside 0..n_nodes-1");
            return GPV_ERR_INVALID;
        }
    const Adjacency adj = build_adjacency(elements, n_elements, nodes_per_element, n_nodes);
    MeshRun R;
    R.solver = solver; R.solver_user = solver_user;
    R.nodes = nodes; R.n = n_nodes; R.mp = mp; R.out = out; R.rounds = rounds;
    R.p_len = 6 * mp->subset_order;
    R.stored.assign(n_nodes, 0);
    R.propagated.assign(n_nodes, 0);
    R.quality_ok.assign(n_nodes, 0);
    R.c_zncc.assign(n_nodes, 0.0);
    R.p.assign(12 * n_nodes, 0.0);
    // seed (src/mesh.rs:667-677): nearest node, forced warp, seed tolerance
    int64_t seed = 0;
    double best = 0.0;
    for (int64_t i = 0; i < n_nodes; i++) {
        const double dx = nodes[2 * i] - mp->seed_coord[0], dy = nodes[2 * i + 1] - mp->seed_coord[1];
        const double d2 = dx * dx + dy * dy;
        if (i == 0 || d2 < best) { best = d2; seed = i; }
    }
    {
        std::vector<double> w(12, 0.0);
        for (int k = 0; k < R.p_len; k++) w[k] = mp->seed_warp[k];
        std::vector<gpv_subset_result> res;
        if (int rc = R.solve_nodes({seed}, {w}, mp->seed_tolerance, res)) return rc;
        if (int rc = R.store(seed, res[0])) return rc;
        R.round++;
        R.propagated[seed] = 1;
        R.push(seed);
    }
    if (!mp->layer_rg) {  // Preconditioning::Rg (:683-705)
        if (int rc = R.neighbours_from(adj, seed)) return rc;
        while (!R.queue.empty()) {
            const int64_t cur = R.queue.top().second;
            R.queue.pop();
            if (R.propagated[cur]) continue;
            R.propagated[cur] = 1;
            if (int rc = R.neighbours_from(adj, cur)) return rc;
        }
    } else {  // Preconditioning::LayerRg (:706-764)
        const int64_t root_cap = (int64_t)mp->batch_factor * mp->max_workers;
        const double eps = mp->root_rel_eps;
        if (int rc = R.expand(adj, {seed})) return rc;
        while (!R.queue.empty()) {
            const auto top = R.queue.top();
            R.queue.pop();
            if (R.propagated[top.second]) continue;
            R.propagated[top.second] = 1;
            std::vector<int64_t> roots = {top.second};
            double top_val;
            std::memcpy(&top_val, &top.first, sizeof top_val);
            const double threshold = top_val * (1.0 - eps);
            while ((int64_t)roots.size() < root_cap && !R.queue.empty()) {
                double k;
                std::memcpy(&k, &R.queue.top().first, sizeof k);
                if (!(k >= threshold)) break;
                const int64_t r = R.queue.top().second;
                R.queue.pop();
                if (R.propagated[r]) continue;
                R.propagated[r] = 1;
                roots.push_back(r);
            }
            if (int rc = R.expand(adj, roots)) return rc;
        }
    }
    gpv_mesh_stats st{};
    st.seed_node = seed;
    for (int64_t i = 0; i < n_nodes; i++) {
        if (!R.stored[i]) {  // a node no propagation reaches is never solved
            std::memset(&out[i], 0, sizeof(out[i]));
            out[i].status = GPV_INVALID_SUBSET;
            if (rounds) rounds[i] = -1;
            st.n_unreached++;
        }
        if (!R.quality_ok[i]) st.n_bad++;  // what the quality gate counts (:792-799)
    }
    st.batches = R.batches;
    st.solves = R.solves;
    st.retries = R.retries;
    st.rounds = R.round;
    if (stats) *stats = st;
    return GPV_SUCCESS;
}

}  // namespace gpv
