/*
 * CPU oracle of the tree-d-3d field solver: a plain-C restatement of the
 * reference's CPU kernels (max-models/tree-d-3d, src/tree_d_3d/kernels/<name>/
 * <name>_pyccel.py), one function per reference kernel, same arguments in the
 * same order, same arithmetic in the same order (built with -ffp-contract=off,
 * so no FMA contraction, as the reference's default Pyccel build).
 *
 * TEST INFRASTRUCTURE ONLY.  It is the checker of the CUDA library and the
 * timed CPU baseline of bench.py; no product code path calls it.
 *
 * Array conventions: component-major points are (2, n) row-major arrays given
 * as a pointer and a row stride (pos[0 * stride + j] is x of particle j);
 * node-major arrays (nodes, k) are row-major with k columns.  Indices are
 * int64.  The OpenMP loops are the reference's `#$ omp parallel for` loops,
 * whose iterations write disjoint outputs, so results do not depend on the
 * thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t i64;

#define MAX(a, b) ((a) > (b) ? (a) : (b))
#define MIN(a, b) ((a) < (b) ? (a) : (b))

/* quadtree_build: K/quadtree_build/quadtree_build_pyccel.py:12-137.
 * sorted_pos (2, n+1 stride), cursor capacity = node array capacity. */
void quadtree_build(double* sorted_pos, i64 spos_stride, i64 n, i64 leaf_capacity,
                    i64 max_depth, double* node_center, double* node_half,
                    i64* node_start, i64* node_end, i64* node_child, i64* node_depth,
                    i64* perm, i64* levels, i64* slot_node, i64* quadrant, i64* cursor,
                    i64 capacity, double* new_sorted_pos, i64 nspos_stride, i64* new_perm,
                    i64* new_slot_node, i64* sizes) {
    for (i64 k = 0; k < n; ++k) {
        perm[k] = k;
        slot_node[k] = 0;
    }
    node_start[0] = 0;
    node_end[0] = n;
    node_depth[0] = 0;
    levels[0] = 0;
    levels[1] = 1;
    i64 n_levels = 1, lo = 0, hi = 1;
    sizes[2] = 0;
    double* sx = sorted_pos;
    double* sy = sorted_pos + spos_stride;
    double* nx = new_sorted_pos;
    double* ny = new_sorted_pos + nspos_stride;
    for (;;) {
        i64 count = hi;
        for (i64 node = lo; node < hi; ++node) {
            if (node_end[node] - node_start[node] > leaf_capacity && node_depth[node] < max_depth) {
                if (count + 4 > capacity) {
                    sizes[2] = 1;
                    return;
                }
                node_child[node] = count;
                double half = 0.5 * node_half[node];
                for (int c = 0; c < 4; ++c) {
                    node_half[count + c] = half;
                    node_depth[count + c] = node_depth[node] + 1;
                    cursor[count + c] = 0;
                }
                double cx = node_center[2 * node], cy = node_center[2 * node + 1];
                node_center[2 * count] = cx - half;
                node_center[2 * count + 1] = cy + half;
                node_center[2 * (count + 1)] = cx + half;
                node_center[2 * (count + 1) + 1] = cy + half;
                node_center[2 * (count + 2)] = cx - half;
                node_center[2 * (count + 2) + 1] = cy - half;
                node_center[2 * (count + 3)] = cx + half;
                node_center[2 * (count + 3) + 1] = cy - half;
                count += 4;
            } else {
                node_child[node] = -1;
            }
        }
        if (count == hi) break;
        for (i64 k = 0; k < n; ++k) {
            i64 node = slot_node[k];
            i64 child = node_child[node];
            if (child < 0) {
                quadrant[k] = -1;
                continue;
            }
            i64 q = 0;
            if (sx[k] > node_center[2 * node]) q += 1;
            if (sy[k] < node_center[2 * node + 1]) q += 2;
            quadrant[k] = q;
            cursor[child + q] += 1;
        }
        for (i64 node = lo; node < hi; ++node) {
            i64 child = node_child[node];
            if (child < 0) continue;
            i64 start = node_start[node];
            for (int q = 0; q < 4; ++q) {
                i64 size = cursor[child + q];
                node_start[child + q] = start;
                node_end[child + q] = start + size;
                cursor[child + q] = start;
                start += size;
            }
        }
        for (i64 k = 0; k < n; ++k) {
            i64 q = quadrant[k], slot;
            if (q < 0) {
                slot = k;
                new_slot_node[slot] = slot_node[k];
            } else {
                i64 child = node_child[slot_node[k]] + q;
                slot = cursor[child];
                cursor[child] += 1;
                new_slot_node[slot] = child;
            }
            new_perm[slot] = perm[k];
            nx[slot] = sx[k];
            ny[slot] = sy[k];
        }
        for (i64 k = 0; k < n; ++k) {
            perm[k] = new_perm[k];
            slot_node[k] = new_slot_node[k];
            sx[k] = nx[k];
            sy[k] = ny[k];
        }
        lo = hi;
        hi = count;
        n_levels += 1;
        levels[n_levels] = hi;
    }
    sizes[0] = hi;
    sizes[1] = n_levels;
}

/* quadtree_moments_upward: K/quadtree_moments_upward/quadtree_moments_upward_pyccel.py:13-83 */
void quadtree_moments_upward(const double* pos, i64 pos_stride, const double* charge,
                             const i64* perm, const i64* levels, i64 n_levels_plus1,
                             const double* node_center, const i64* node_start,
                             const i64* node_end, const i64* node_child, double* node_q,
                             double* node_qabs, double* node_p, double* node_s) {
    i64 n_levels = n_levels_plus1 - 1;
    for (i64 level = n_levels - 1; level >= 0; --level) {
#pragma omp parallel for schedule(dynamic, 64)
        for (i64 node = levels[level]; node < levels[level + 1]; ++node) {
            double q = 0.0, qabs = 0.0, px = 0.0, py = 0.0, sxx = 0.0, sxy = 0.0, syy = 0.0;
            double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
            i64 first = node_child[node];
            if (first < 0) {
                for (i64 k = node_start[node]; k < node_end[node]; ++k) {
                    i64 j = perm[k];
                    double c = charge[j];
                    double dx = pos[j] - xmid;
                    double dy = pos[pos_stride + j] - ymid;
                    q += c;
                    qabs += fabs(c);
                    px += c * dx;
                    py += c * dy;
                    sxx += c * dx * dx;
                    sxy += c * dx * dy;
                    syy += c * dy * dy;
                }
            } else {
                for (i64 child = first; child < first + 4; ++child) {
                    double dx = node_center[2 * child] - xmid;
                    double dy = node_center[2 * child + 1] - ymid;
                    double cq = node_q[child], cpx = node_p[2 * child], cpy = node_p[2 * child + 1];
                    q += cq;
                    qabs += node_qabs[child];
                    px += cpx + cq * dx;
                    py += cpy + cq * dy;
                    sxx += node_s[3 * child] + 2.0 * cpx * dx + cq * dx * dx;
                    sxy += node_s[3 * child + 1] + cpx * dy + cpy * dx + cq * dx * dy;
                    syy += node_s[3 * child + 2] + 2.0 * cpy * dy + cq * dy * dy;
                }
            }
            node_q[node] = q;
            node_qabs[node] = qabs;
            node_p[2 * node] = px;
            node_p[2 * node + 1] = py;
            node_s[3 * node] = sxx;
            node_s[3 * node + 1] = sxy;
            node_s[3 * node + 2] = syy;
        }
    }
}

/* log_moments_upward: K/log_moments_upward/log_moments_upward_pyccel.py:14-93.
 * binomial is (bsize, bsize) row-major. */
void log_moments_upward(const double* pos, i64 pos_stride, const double* charge,
                        const i64* perm, const i64* levels, i64 n_levels_plus1,
                        const double* node_center, const i64* node_start, const i64* node_end,
                        const i64* node_child, const double* binomial, i64 bsize,
                        double* node_qabs, double* moment_re, double* moment_im, i64 order) {
    i64 n_levels = n_levels_plus1 - 1;
    i64 w = order + 1;
    for (i64 level = n_levels - 1; level >= 0; --level) {
#pragma omp parallel for schedule(dynamic, 64)
        for (i64 node = levels[level]; node < levels[level + 1]; ++node) {
            double sh_re[129], sh_im[129];
            double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
            double* mre = moment_re + node * w;
            double* mim = moment_im + node * w;
            for (i64 n = 0; n <= order; ++n) {
                mre[n] = 0.0;
                mim[n] = 0.0;
            }
            i64 first = node_child[node];
            if (first < 0) {
                double qabs = 0.0;
                for (i64 k = node_start[node]; k < node_end[node]; ++k) {
                    i64 j = perm[k];
                    double q = charge[j];
                    qabs += fabs(q);
                    double dx = pos[j] - xmid, dy = pos[pos_stride + j] - ymid;
                    double pr = q, pi = 0.0;
                    for (i64 n = 0; n <= order; ++n) {
                        mre[n] += pr;
                        mim[n] += pi;
                        double next_re = pr * dx - pi * dy;
                        pi = pr * dy + pi * dx;
                        pr = next_re;
                    }
                }
                node_qabs[node] = qabs;
            } else {
                double qabs = 0.0;
                for (i64 child = first; child < first + 4; ++child) {
                    qabs += node_qabs[child];
                    if (node_end[child] == node_start[child]) continue;
                    double s_re = node_center[2 * child] - xmid;
                    double s_im = node_center[2 * child + 1] - ymid;
                    sh_re[0] = 1.0;
                    sh_im[0] = 0.0;
                    for (i64 n = 1; n <= order; ++n) {
                        sh_re[n] = sh_re[n - 1] * s_re - sh_im[n - 1] * s_im;
                        sh_im[n] = sh_re[n - 1] * s_im + sh_im[n - 1] * s_re;
                    }
                    const double* cre = moment_re + child * w;
                    const double* cim = moment_im + child * w;
                    for (i64 n = 0; n <= order; ++n) {
                        double acc_re = 0.0, acc_im = 0.0;
                        for (i64 m = 0; m <= n; ++m) {
                            double c = binomial[n * bsize + m];
                            double a_re = cre[m] * c, a_im = cim[m] * c;
                            acc_re += a_re * sh_re[n - m] - a_im * sh_im[n - m];
                            acc_im += a_re * sh_im[n - m] + a_im * sh_re[n - m];
                        }
                        mre[n] += acc_re;
                        mim[n] += acc_im;
                    }
                }
                node_qabs[node] = qabs;
            }
        }
    }
}

/* evaluate_quadtree: K/evaluate_quadtree/evaluate_quadtree_pyccel.py:17-152
 * (the per-target walk; the reference's grouped CPU walk evaluate_groups,
 * K/evaluate_groups/evaluate_groups_pyccel.py:16-297, gives each target the
 * same terms in the same order). */
void evaluate_quadtree(const double* targets, i64 t_stride, i64 num_targets, const i64* exclude,
                       const double* pos, i64 pos_stride, const double* charge, const i64* perm,
                       const double* node_center, const double* node_half,
                       const i64* node_start, const i64* node_end, const i64* node_child,
                       const double* node_q, const double* node_qabs, const double* node_p,
                       const double* node_s, double theta, double softening, i64 stack_size,
                       int with_potential, double* phi, double* field, i64 f_stride,
                       i64* status) {
    double eps2 = softening * softening;
    i64 num_bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : num_bad)
    for (i64 i = 0; i < num_targets; ++i) {
        i64* walk = (i64*)malloc(sizeof(i64) * stack_size);
        double tx = targets[i], ty = targets[t_stride + i];
        i64 skip = exclude[i];
        int bad = 0;
        double potential = 0.0, ex = 0.0, ey = 0.0;
        walk[0] = 0;
        i64 top = 1;
        while (top > 0) {
            top -= 1;
            i64 node = walk[top];
            if (node_qabs[node] == 0.0) continue;
            i64 first = node_child[node];
            if (first < 0) {
                for (i64 k = node_start[node]; k < node_end[node]; ++k) {
                    i64 j = perm[k];
                    double c = charge[j];
                    if (j == skip || c == 0.0) continue;
                    double dx = tx - pos[j], dy = ty - pos[pos_stride + j];
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad = 1;
                        break;
                    }
                    double inv_r = 1.0 / sqrt(r2);
                    double inv_r3 = inv_r * inv_r * inv_r;
                    potential += c * inv_r;
                    ex += c * inv_r3 * dx;
                    ey += c * inv_r3 * dy;
                }
                if (bad) top = 0;
                continue;
            }
            double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
            double half = node_half[node];
            double rx = tx - xmid, ry = ty - ymid;
            double distance = sqrt(rx * rx + ry * ry);
            int inside = tx >= xmid - half && tx <= xmid + half && ty >= ymid - half &&
                         ty <= ymid + half;
            if (!inside && 2.0 * half < theta * distance) {
                double inv_r = 1.0 / sqrt(distance * distance + eps2);
                double inv_r2 = inv_r * inv_r;
                double inv_r3 = inv_r2 * inv_r;
                double inv_r5 = inv_r3 * inv_r2;
                double inv_r7 = inv_r5 * inv_r2;
                double q = node_q[node], px = node_p[2 * node], py = node_p[2 * node + 1];
                double sxx = node_s[3 * node], sxy = node_s[3 * node + 1],
                       syy = node_s[3 * node + 2];
                double pr = px * rx + py * ry;
                double srx = sxx * rx + sxy * ry;
                double sry = sxy * rx + syy * ry;
                double rsr = rx * srx + ry * sry;
                double trace = sxx + syy;
                potential += q * inv_r + pr * inv_r3 + 0.5 * (3.0 * rsr * inv_r5 - trace * inv_r3);
                double radial = q * inv_r3 + 3.0 * pr * inv_r5 + 7.5 * rsr * inv_r7 -
                                1.5 * trace * inv_r5;
                ex += radial * rx - px * inv_r3 - 3.0 * srx * inv_r5;
                ey += radial * ry - py * inv_r3 - 3.0 * sry * inv_r5;
            } else {
                for (int child = 0; child < 4; ++child) {
                    walk[top] = first + child;
                    top += 1;
                }
            }
        }
        free(walk);
        if (bad) {
            num_bad += 1;
            phi[i] = 1.0e300;
        } else {
            phi[i] = with_potential ? potential : 0.0;
            field[i] = ex;
            field[f_stride + i] = ey;
        }
    }
    if (num_bad > 0) {
        for (i64 i = 0; i < num_targets; ++i) {
            if (phi[i] == 1.0e300) {
                phi[i] = 0.0;
                status[0] = i + 1;
                return;
            }
        }
    }
}

/* evaluate_log_quadtree: K/evaluate_log_quadtree/evaluate_log_quadtree_pyccel.py:17-150;
 * with_potential = 0 skips the logarithms as evaluate_groups_pyccel.py:115-116,:218-219. */
void evaluate_log_quadtree(const double* targets, i64 t_stride, i64 num_targets,
                           const i64* exclude, const double* pos, i64 pos_stride,
                           const double* charge, const i64* perm, const double* node_center,
                           const double* node_half, const i64* node_start,
                           const i64* node_end, const i64* node_child,
                           const double* node_qabs, const double* moment_re,
                           const double* moment_im, i64 order, double theta, double softening,
                           i64 stack_size, int with_potential, double* phi, double* field,
                           i64 f_stride, i64* status) {
    double eps2 = softening * softening;
    i64 num_bad = 0;
    i64 w = order + 1;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : num_bad)
    for (i64 i = 0; i < num_targets; ++i) {
        i64* walk = (i64*)malloc(sizeof(i64) * stack_size);
        double tx = targets[i], ty = targets[t_stride + i];
        i64 skip = exclude[i];
        int bad = 0;
        double potential = 0.0, ex = 0.0, ey = 0.0;
        walk[0] = 0;
        i64 top = 1;
        while (top > 0) {
            top -= 1;
            i64 node = walk[top];
            if (node_qabs[node] == 0.0) continue;
            i64 first = node_child[node];
            if (first < 0) {
                for (i64 k = node_start[node]; k < node_end[node]; ++k) {
                    i64 j = perm[k];
                    double c = charge[j];
                    if (j == skip || c == 0.0) continue;
                    double dx = tx - pos[j], dy = ty - pos[pos_stride + j];
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad = 1;
                        break;
                    }
                    if (with_potential) potential -= c * log(r2);
                    ex += 2.0 * c * dx / r2;
                    ey += 2.0 * c * dy / r2;
                }
                if (bad) top = 0;
                continue;
            }
            double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
            double half = node_half[node];
            double rx = tx - xmid, ry = ty - ymid;
            double d2 = rx * rx + ry * ry;
            int inside = tx >= xmid - half && tx <= xmid + half && ty >= ymid - half &&
                         ty <= ymid + half;
            if (!inside && 4.0 * half * half < theta * theta * d2) {
                double w_re = rx / d2, w_im = -ry / d2;
                double prev_re = 1.0, prev_im = 0.0, cur_re = w_re, cur_im = w_im;
                double f_re = 0.0, f_im = 0.0, series = 0.0;
                const double* are = moment_re + node * w;
                const double* aim = moment_im + node * w;
                for (i64 n = 0; n <= order; ++n) {
                    double a_re = are[n], a_im = aim[n];
                    f_re += a_re * cur_re - a_im * cur_im;
                    f_im += a_re * cur_im + a_im * cur_re;
                    if (n > 0) series += (a_re * prev_re - a_im * prev_im) / (double)n;
                    prev_re = cur_re;
                    prev_im = cur_im;
                    double next_re = cur_re * w_re - cur_im * w_im;
                    cur_im = cur_re * w_im + cur_im * w_re;
                    cur_re = next_re;
                }
                if (with_potential) potential += -are[0] * log(d2) + 2.0 * series;
                ex += 2.0 * f_re;
                ey -= 2.0 * f_im;
            } else {
                for (int child = 0; child < 4; ++child) {
                    walk[top] = first + child;
                    top += 1;
                }
            }
        }
        free(walk);
        if (bad) {
            num_bad += 1;
            phi[i] = 1.0e300;
        } else {
            phi[i] = potential;
            field[i] = ex;
            field[f_stride + i] = ey;
        }
    }
    if (num_bad > 0) {
        for (i64 i = 0; i < num_targets; ++i) {
            if (phi[i] == 1.0e300) {
                phi[i] = 0.0;
                status[0] = i + 1;
                return;
            }
        }
    }
}

/* direct_sum: K/direct_sum/direct_sum_pyccel.py:15-72 */
void direct_sum(const double* targets, i64 t_stride, i64 num_targets, const i64* exclude,
                const double* pos, i64 pos_stride, i64 num_sources, const double* charge,
                double softening, double* phi, double* field, i64 f_stride, i64* status) {
    double eps2 = softening * softening;
    i64 num_bad = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : num_bad)
    for (i64 i = 0; i < num_targets; ++i) {
        double tx = targets[i], ty = targets[t_stride + i];
        i64 skip = exclude[i];
        double potential = 0.0, ex = 0.0, ey = 0.0;
        int bad = 0;
        for (i64 j = 0; j < num_sources; ++j) {
            double c = charge[j];
            if (j == skip || c == 0.0) continue;
            double dx = tx - pos[j], dy = ty - pos[pos_stride + j];
            double r2 = dx * dx + dy * dy + eps2;
            if (r2 == 0.0) {
                bad = 1;
                break;
            }
            double inv_r = 1.0 / sqrt(r2);
            double inv_r3 = inv_r * inv_r * inv_r;
            potential += c * inv_r;
            ex += c * inv_r3 * dx;
            ey += c * inv_r3 * dy;
        }
        if (bad) {
            num_bad += 1;
            phi[i] = 1.0e300;
        } else {
            phi[i] = potential;
            field[i] = ex;
            field[f_stride + i] = ey;
        }
    }
    if (num_bad > 0) {
        for (i64 i = 0; i < num_targets; ++i) {
            if (phi[i] == 1.0e300) {
                phi[i] = 0.0;
                status[0] = i + 1;
                return;
            }
        }
    }
}

/* direct_log_sum: K/direct_log_sum/direct_log_sum_pyccel.py:15-70 */
void direct_log_sum(const double* targets, i64 t_stride, i64 num_targets, const i64* exclude,
                    const double* pos, i64 pos_stride, i64 num_sources, const double* charge,
                    double softening, double* phi, double* field, i64 f_stride, i64* status) {
    double eps2 = softening * softening;
    i64 num_bad = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : num_bad)
    for (i64 i = 0; i < num_targets; ++i) {
        double tx = targets[i], ty = targets[t_stride + i];
        i64 skip = exclude[i];
        double potential = 0.0, ex = 0.0, ey = 0.0;
        int bad = 0;
        for (i64 j = 0; j < num_sources; ++j) {
            double c = charge[j];
            if (j == skip || c == 0.0) continue;
            double dx = tx - pos[j], dy = ty - pos[pos_stride + j];
            double r2 = dx * dx + dy * dy + eps2;
            if (r2 == 0.0) {
                bad = 1;
                break;
            }
            potential -= c * log(r2);
            ex += 2.0 * c * dx / r2;
            ey += 2.0 * c * dy / r2;
        }
        if (bad) {
            num_bad += 1;
            phi[i] = 1.0e300;
        } else {
            phi[i] = potential;
            field[i] = ex;
            field[f_stride + i] = ey;
        }
    }
    if (num_bad > 0) {
        for (i64 i = 0; i < num_targets; ++i) {
            if (phi[i] == 1.0e300) {
                phi[i] = 0.0;
                status[0] = i + 1;
                return;
            }
        }
    }
}

/* pair_energy: K/pair_energy/pair_energy_pyccel.py:15-60 */
void pair_energy(const double* pos, i64 pos_stride, i64 n, const double* charge,
                 double softening, i64* status, double* energy) {
    double eps2 = softening * softening;
    double total = 0.0;
    i64 num_bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total, num_bad)
    for (i64 i = 0; i < n; ++i) {
        double ci = charge[i];
        if (ci == 0.0) continue;
        double partial = 0.0;
        int bad = 0;
        for (i64 j = i + 1; j < n; ++j) {
            double cj = charge[j];
            if (cj == 0.0) continue;
            double dx = pos[i] - pos[j], dy = pos[pos_stride + i] - pos[pos_stride + j];
            double r2 = dx * dx + dy * dy + eps2;
            if (r2 == 0.0) {
                bad = 1;
                break;
            }
            partial += cj / sqrt(r2);
        }
        if (bad)
            num_bad += 1;
        else
            total += ci * partial;
    }
    if (num_bad > 0) {
        status[0] = 1;
        return;
    }
    energy[0] += total;
}

/* fmm_traverse: K/fmm_traverse/fmm_traverse_pyccel.py:15-106 (one generation).
 * frontier / next_frontier / m2l / p2p are (capacity, 2) row-major. */
void fmm_traverse(const double* node_center, const double* node_half, const i64* node_start,
                  const i64* node_end, const i64* node_child, double theta, const i64* frontier,
                  i64 n_frontier, i64* next_frontier, i64 next_cap, i64* m2l, i64 m2l_cap,
                  i64* p2p, i64 p2p_cap, i64* counts) {
    double root2 = sqrt(2.0);
    for (i64 k = 0; k < n_frontier; ++k) {
        i64 a = frontier[2 * k], b = frontier[2 * k + 1];
        if (node_end[a] == node_start[a] || node_end[b] == node_start[b]) continue;
        int leaf_a = node_child[a] < 0, leaf_b = node_child[b] < 0;
        if (a == b) {
            if (leaf_a) {
                i64 i = counts[1];
                counts[1] = i + 1;
                if (i < p2p_cap) {
                    p2p[2 * i] = a;
                    p2p[2 * i + 1] = a;
                } else {
                    counts[3] = -1;
                }
                continue;
            }
            i64 first = node_child[a];
            i64 i = counts[2];
            counts[2] = i + 10;
            if (i + 10 > next_cap) {
                counts[3] = -1;
                continue;
            }
            for (int c = 0; c < 4; ++c)
                for (int d = c; d < 4; ++d) {
                    next_frontier[2 * i] = first + c;
                    next_frontier[2 * i + 1] = first + d;
                    i += 1;
                }
            continue;
        }
        double dx = node_center[2 * a] - node_center[2 * b];
        double dy = node_center[2 * a + 1] - node_center[2 * b + 1];
        double distance = sqrt(dx * dx + dy * dy);
        double radii = root2 * (node_half[a] + node_half[b]);
        if (radii < theta * distance) {
            i64 i = counts[0];
            counts[0] = i + 1;
            if (i < m2l_cap) {
                m2l[2 * i] = a;
                m2l[2 * i + 1] = b;
            } else {
                counts[3] = -1;
            }
            continue;
        }
        if (leaf_a && leaf_b) {
            i64 i = counts[1];
            counts[1] = i + 1;
            if (i < p2p_cap) {
                p2p[2 * i] = a;
                p2p[2 * i + 1] = b;
            } else {
                counts[3] = -1;
            }
            continue;
        }
        i64 i = counts[2];
        counts[2] = i + 4;
        if (i + 4 > next_cap) {
            counts[3] = -1;
            continue;
        }
        if (leaf_b || (!leaf_a && node_half[a] >= node_half[b])) {
            i64 first = node_child[a];
            for (int c = 0; c < 4; ++c) {
                next_frontier[2 * (i + c)] = first + c;
                next_frontier[2 * (i + c) + 1] = b;
            }
        } else {
            i64 first = node_child[b];
            for (int c = 0; c < 4; ++c) {
                next_frontier[2 * (i + c)] = a;
                next_frontier[2 * (i + c) + 1] = first + c;
            }
        }
    }
}

/* pair_csr: K/pair_csr/pair_csr_pyccel.py:12-45.  row_start (n_nodes + 1) zero on entry. */
void pair_csr(const i64* pairs, i64 count, int mutual, i64* row_start, i64 n_nodes,
              i64* partner, i64* cursor) {
    for (i64 p = 0; p < count; ++p) {
        i64 a = pairs[2 * p], b = pairs[2 * p + 1];
        row_start[a + 1] += 1;
        if (mutual && a != b) row_start[b + 1] += 1;
    }
    for (i64 n = 0; n < n_nodes; ++n) {
        row_start[n + 1] += row_start[n];
        cursor[n] = row_start[n];
    }
    for (i64 p = 0; p < count; ++p) {
        i64 a = pairs[2 * p], b = pairs[2 * p + 1];
        partner[cursor[a]] = b;
        cursor[a] += 1;
        if (mutual && a != b) {
            partner[cursor[b]] = a;
            cursor[b] += 1;
        }
    }
}

/* fmm_m2l_host: K/fmm_m2l_host/fmm_m2l_host_pyccel.py:16-105.
 * coeff (order+1, order+1) row-major; locals/moments (nodes, order+1). */
void fmm_m2l_host(const i64* row_start, i64 n_nodes, const i64* sources,
                  const double* dst_center, const double* src_center, const double* moment_re,
                  const double* moment_im, const double* coeff, double* local_re,
                  double* local_im, i64 order) {
    i64 w = order + 1;
    i64 n_chunks = (n_nodes + 63) / 64;
#pragma omp parallel for schedule(dynamic, 1)
    for (i64 chunk = 0; chunk < n_chunks; ++chunk) {
        double b_re[129], b_im[129], s_re[129], s_im[129], pw_re[129], pw_im[129];
        for (i64 dst = 64 * chunk; dst < MIN(64 * chunk + 64, n_nodes); ++dst) {
            if (row_start[dst + 1] == row_start[dst]) continue;
            for (i64 l = 0; l <= order; ++l) b_re[l] = b_im[l] = 0.0;
            double cx = dst_center[2 * dst], cy = dst_center[2 * dst + 1];
            for (i64 e = row_start[dst]; e < row_start[dst + 1]; ++e) {
                i64 src = sources[e];
                double t_re = cx - src_center[2 * src], t_im = cy - src_center[2 * src + 1];
                double t2 = t_re * t_re + t_im * t_im;
                double w_re = t_re / t2, w_im = -t_im / t2;
                pw_re[0] = 1.0;
                pw_im[0] = 0.0;
                for (i64 k = 1; k <= order; ++k) {
                    pw_re[k] = pw_re[k - 1] * w_re - pw_im[k - 1] * w_im;
                    pw_im[k] = pw_re[k - 1] * w_im + pw_im[k - 1] * w_re;
                }
                for (i64 l = 0; l <= order; ++l) s_re[l] = s_im[l] = 0.0;
                for (i64 k = 0; k <= order; ++k) {
                    double a_re = moment_re[src * w + k], a_im = moment_im[src * w + k];
                    double ar = a_re * pw_re[k] - a_im * pw_im[k];
                    double ai = a_re * pw_im[k] + a_im * pw_re[k];
                    for (i64 l = 0; l <= order; ++l) {
                        double c = coeff[k * w + l];
                        s_re[l] += c * ar;
                        s_im[l] += c * ai;
                    }
                }
                double a_re = moment_re[src * w], a_im = moment_im[src * w];
                double log_re = 0.5 * log(t2), log_im = atan2(t_im, t_re);
                b_re[0] += a_re * log_re - a_im * log_im - s_re[0];
                b_im[0] += a_re * log_im + a_im * log_re - s_im[0];
                double sign = 1.0;
                for (i64 l = 1; l <= order; ++l) {
                    b_re[l] += sign * (s_re[l] * pw_re[l] - s_im[l] * pw_im[l]);
                    b_im[l] += sign * (s_re[l] * pw_im[l] + s_im[l] * pw_re[l]);
                    sign = -sign;
                }
            }
            for (i64 l = 0; l <= order; ++l) {
                local_re[dst * w + l] += b_re[l];
                local_im[dst * w + l] += b_im[l];
            }
        }
    }
}

/* fmm_downward: K/fmm_downward/fmm_downward_pyccel.py:15-64 (one level). */
void fmm_downward(i64 first_node, i64 last_node, const double* node_center,
                  const i64* node_child, const double* binomial, i64 bsize, double* local_re,
                  double* local_im, i64 order) {
    i64 w = order + 1;
#pragma omp parallel for schedule(dynamic, 16)
    for (i64 node = first_node; node < last_node; ++node) {
        double sh_re[129], sh_im[129];
        i64 first = node_child[node];
        if (first < 0) continue;
        for (i64 child = first; child < first + 4; ++child) {
            double s_re = node_center[2 * child] - node_center[2 * node];
            double s_im = node_center[2 * child + 1] - node_center[2 * node + 1];
            sh_re[0] = 1.0;
            sh_im[0] = 0.0;
            for (i64 k = 1; k <= order; ++k) {
                sh_re[k] = sh_re[k - 1] * s_re - sh_im[k - 1] * s_im;
                sh_im[k] = sh_re[k - 1] * s_im + sh_im[k - 1] * s_re;
            }
            for (i64 m = 0; m <= order; ++m) {
                double acc_re = 0.0, acc_im = 0.0;
                for (i64 l = m; l <= order; ++l) {
                    double c = binomial[l * bsize + m];
                    double b_re = local_re[node * w + l] * c;
                    double b_im = local_im[node * w + l] * c;
                    acc_re += b_re * sh_re[l - m] - b_im * sh_im[l - m];
                    acc_im += b_re * sh_im[l - m] + b_im * sh_re[l - m];
                }
                local_re[child * w + m] += acc_re;
                local_im[child * w + m] += acc_im;
            }
        }
    }
}

/* fmm_evaluate_host: K/fmm_evaluate_host/fmm_evaluate_host_pyccel.py:14-100.
 * L2P in parallel over leaves, the mutual P2P serial (as the reference). */
void fmm_evaluate_host(const double* spos, i64 sp_stride, const double* scharge,
                       i64 node_count, const double* node_center, const i64* node_start,
                       const i64* node_end, const i64* node_child, const double* local_re,
                       const double* local_im, i64 order, const i64* pairs, i64 count,
                       double softening, int with_potential, double* phi, double* field,
                       i64 f_stride, i64* status) {
    i64 w = order + 1;
    double eps2 = softening * softening;
#pragma omp parallel for schedule(dynamic, 16)
    for (i64 node = 0; node < node_count; ++node) {
        if (node_child[node] >= 0) continue;
        for (i64 k = node_start[node]; k < node_end[node]; ++k) {
            double u_re = spos[k] - node_center[2 * node];
            double u_im = spos[sp_stride + k] - node_center[2 * node + 1];
            double w_re = local_re[node * w + order], w_im = local_im[node * w + order];
            double d_re = 0.0, d_im = 0.0;
            for (i64 l = order - 1; l >= 0; --l) {
                double nd_re = d_re * u_re - d_im * u_im + w_re;
                d_im = d_re * u_im + d_im * u_re + w_im;
                d_re = nd_re;
                double nw_re = w_re * u_re - w_im * u_im + local_re[node * w + l];
                w_im = w_re * u_im + w_im * u_re + local_im[node * w + l];
                w_re = nw_re;
            }
            phi[k] += -2.0 * w_re;
            field[k] += 2.0 * d_re;
            field[f_stride + k] -= 2.0 * d_im;
        }
    }
    for (i64 pair = 0; pair < count; ++pair) {
        i64 a = pairs[2 * pair], b = pairs[2 * pair + 1];
        for (i64 ka = node_start[a]; ka < node_end[a]; ++ka) {
            double xi = spos[ka], yi = spos[sp_stride + ka], qi = scharge[ka];
            double pi = 0.0, fxi = 0.0, fyi = 0.0;
            i64 start_b = node_start[b];
            if (a == b) start_b = ka + 1;
            for (i64 kb = start_b; kb < node_end[b]; ++kb) {
                double qj = scharge[kb];
                double dx = xi - spos[kb], dy = yi - spos[sp_stride + kb];
                double r2 = dx * dx + dy * dy + eps2;
                if (r2 == 0.0) {
                    if (qi != 0.0 && qj != 0.0) {
                        status[0] = ka + 1;
                        return;
                    }
                    continue;
                }
                if (with_potential) {
                    double log_r2 = log(r2);
                    pi -= qj * log_r2;
                    phi[kb] -= qi * log_r2;
                }
                double inv = 2.0 / r2;
                double fx = dx * inv, fy = dy * inv;
                fxi += qj * fx;
                fyi += qj * fy;
                field[kb] -= qi * fx;
                field[f_stride + kb] -= qi * fy;
            }
            phi[ka] += pi;
            field[ka] += fxi;
            field[f_stride + ka] += fyi;
        }
    }
}

/* cart_moments_upward: K/cart_moments_upward/cart_moments_upward_pyccel.py:14-82.
 * shift (n_shift, 3) rows; moments (nodes, n_coef). */
void cart_moments_upward(const double* pos, i64 pos_stride, const double* charge,
                         const i64* perm, const i64* levels, i64 n_levels_plus1,
                         const double* node_center, const i64* node_start, const i64* node_end,
                         const i64* node_child, const i64* mono_parent, const i64* mono_dir,
                         const i64* shift, const double* shift_coef, i64 n_shift,
                         double* moments, i64 n_coef) {
    i64 n_levels = n_levels_plus1 - 1;
    for (i64 level = n_levels - 1; level >= 0; --level) {
#pragma omp parallel for schedule(dynamic, 64)
        for (i64 node = levels[level]; node < levels[level + 1]; ++node) {
            double mono[2145];
            double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
            double* m = moments + node * n_coef;
            for (i64 i = 0; i < n_coef; ++i) m[i] = 0.0;
            i64 first = node_child[node];
            if (first < 0) {
                for (i64 k = node_start[node]; k < node_end[node]; ++k) {
                    i64 j = perm[k];
                    mono[0] = charge[j];
                    for (i64 i = 1; i < n_coef; ++i) {
                        if (mono_dir[i] == 0)
                            mono[i] = mono[mono_parent[i]] * (pos[j] - xmid);
                        else
                            mono[i] = mono[mono_parent[i]] * (pos[pos_stride + j] - ymid);
                    }
                    for (i64 i = 0; i < n_coef; ++i) m[i] += mono[i];
                }
            } else {
                for (i64 child = first; child < first + 4; ++child) {
                    if (node_end[child] == node_start[child]) continue;
                    mono[0] = 1.0;
                    for (i64 i = 1; i < n_coef; ++i) {
                        if (mono_dir[i] == 0)
                            mono[i] = mono[mono_parent[i]] * (node_center[2 * child] - xmid);
                        else
                            mono[i] = mono[mono_parent[i]] * (node_center[2 * child + 1] - ymid);
                    }
                    const double* cm = moments + child * n_coef;
                    for (i64 t = 0; t < n_shift; ++t)
                        m[shift[3 * t]] += shift_coef[t] * cm[shift[3 * t + 1]] * mono[shift[3 * t + 2]];
                }
            }
        }
    }
}

/* cart_m2l_host: K/cart_m2l_host/cart_m2l_host_pyccel.py:16-80. rec (n_coef, 4), m2l (n_terms, 3). */
void cart_m2l_host(const i64* row_start, i64 n_nodes, const i64* sources,
                   const double* dst_center, const double* src_center, const double* moments,
                   i64 n_coef, double softening, const i64* ex, const i64* ey, const i64* rec,
                   const i64* m2l, const double* m2l_coef, i64 n_terms, double* local) {
    double eps2 = softening * softening;
    i64 n_chunks = (n_nodes + 63) / 64;
#pragma omp parallel for schedule(dynamic, 1)
    for (i64 chunk = 0; chunk < n_chunks; ++chunk) {
        double acc[2145], coef[2145];
        for (i64 dst = 64 * chunk; dst < MIN(64 * chunk + 64, n_nodes); ++dst) {
            if (row_start[dst + 1] == row_start[dst]) continue;
            for (i64 i = 0; i < n_coef; ++i) acc[i] = 0.0;
            double cx = dst_center[2 * dst], cy = dst_center[2 * dst + 1];
            for (i64 e = row_start[dst]; e < row_start[dst + 1]; ++e) {
                i64 src = sources[e];
                double tx = cx - src_center[2 * src], ty = cy - src_center[2 * src + 1];
                double r2 = tx * tx + ty * ty + eps2;
                coef[0] = 1.0 / sqrt(r2);
                for (i64 i = 1; i < n_coef; ++i) {
                    i64 n = ex[i] + ey[i];
                    double s = 0.0;
                    if (rec[4 * i] >= 0) s += (double)(2 * n - 1) * tx * coef[rec[4 * i]];
                    if (rec[4 * i + 1] >= 0) s += (double)(2 * n - 1) * ty * coef[rec[4 * i + 1]];
                    if (rec[4 * i + 2] >= 0) s += (double)(n - 1) * coef[rec[4 * i + 2]];
                    if (rec[4 * i + 3] >= 0) s += (double)(n - 1) * coef[rec[4 * i + 3]];
                    coef[i] = -s / ((double)n * r2);
                }
                const double* ms = moments + src * n_coef;
                for (i64 t = 0; t < n_terms; ++t)
                    acc[m2l[3 * t]] += m2l_coef[t] * ms[m2l[3 * t + 1]] * coef[m2l[3 * t + 2]];
            }
            for (i64 i = 0; i < n_coef; ++i) local[dst * n_coef + i] += acc[i];
        }
    }
}

/* cart_downward: K/cart_downward/cart_downward_pyccel.py:14-55 */
void cart_downward(const i64* levels, i64 n_levels_plus1, const double* node_center,
                   const i64* node_child, const i64* mono_parent, const i64* mono_dir,
                   const i64* shift, const double* shift_coef, i64 n_shift, double* local,
                   i64 n_coef) {
    i64 n_levels = n_levels_plus1 - 1;
    for (i64 level = 0; level < n_levels - 1; ++level) {
#pragma omp parallel for schedule(dynamic, 16)
        for (i64 node = levels[level]; node < levels[level + 1]; ++node) {
            double mono[2145];
            i64 first = node_child[node];
            if (first < 0) continue;
            for (i64 child = first; child < first + 4; ++child) {
                mono[0] = 1.0;
                for (i64 i = 1; i < n_coef; ++i) {
                    if (mono_dir[i] == 0)
                        mono[i] = mono[mono_parent[i]] * (node_center[2 * child] - node_center[2 * node]);
                    else
                        mono[i] = mono[mono_parent[i]] *
                                  (node_center[2 * child + 1] - node_center[2 * node + 1]);
                }
                for (i64 t = 0; t < n_shift; ++t)
                    local[child * n_coef + shift[3 * t + 1]] +=
                        shift_coef[t] * local[node * n_coef + shift[3 * t]] * mono[shift[3 * t + 2]];
            }
        }
    }
}

/* cart_evaluate_host: K/cart_evaluate_host/cart_evaluate_host_pyccel.py:16-110 */
void cart_evaluate_host(const double* spos, i64 sp_stride, const double* scharge,
                        i64 node_count, const double* node_center, const i64* node_start,
                        const i64* node_end, const i64* node_child, const double* local,
                        i64 n_coef, const i64* mono_parent, const i64* mono_dir, const i64* ex,
                        const i64* ey, const i64* grad, const i64* pairs, i64 count,
                        double softening, double* phi, double* field, i64 f_stride,
                        i64* status) {
    double eps2 = softening * softening;
#pragma omp parallel for schedule(dynamic, 16)
    for (i64 node = 0; node < node_count; ++node) {
        double mono[2145];
        if (node_child[node] >= 0) continue;
        const double* L = local + node * n_coef;
        for (i64 k = node_start[node]; k < node_end[node]; ++k) {
            mono[0] = 1.0;
            for (i64 i = 1; i < n_coef; ++i) {
                if (mono_dir[i] == 0)
                    mono[i] = mono[mono_parent[i]] * (spos[k] - node_center[2 * node]);
                else
                    mono[i] = mono[mono_parent[i]] * (spos[sp_stride + k] - node_center[2 * node + 1]);
            }
            double wv = 0.0, gx = 0.0, gy = 0.0;
            for (i64 i = 0; i < n_coef; ++i) {
                wv += L[i] * mono[i];
                if (grad[2 * i] >= 0) gx += (double)ex[i] * L[i] * mono[grad[2 * i]];
                if (grad[2 * i + 1] >= 0) gy += (double)ey[i] * L[i] * mono[grad[2 * i + 1]];
            }
            phi[k] += wv;
            field[k] -= gx;
            field[f_stride + k] -= gy;
        }
    }
    for (i64 pair = 0; pair < count; ++pair) {
        i64 a = pairs[2 * pair], b = pairs[2 * pair + 1];
        for (i64 ka = node_start[a]; ka < node_end[a]; ++ka) {
            double xi = spos[ka], yi = spos[sp_stride + ka], qi = scharge[ka];
            double pi = 0.0, fxi = 0.0, fyi = 0.0;
            i64 start_b = node_start[b];
            if (a == b) start_b = ka + 1;
            for (i64 kb = start_b; kb < node_end[b]; ++kb) {
                double qj = scharge[kb];
                double dx = xi - spos[kb], dy = yi - spos[sp_stride + kb];
                double r2 = dx * dx + dy * dy + eps2;
                if (r2 == 0.0) {
                    if (qi != 0.0 && qj != 0.0) {
                        status[0] = ka + 1;
                        return;
                    }
                    continue;
                }
                double inv_r = 1.0 / sqrt(r2);
                double inv_r3 = inv_r * inv_r * inv_r;
                pi += qj * inv_r;
                phi[kb] += qi * inv_r;
                fxi += qj * inv_r3 * dx;
                fyi += qj * inv_r3 * dy;
                field[kb] -= qi * inv_r3 * dx;
                field[f_stride + kb] -= qi * inv_r3 * dy;
            }
            phi[ka] += pi;
            field[ka] += fxi;
            field[f_stride + ka] += fyi;
        }
    }
}

/* dual_traverse: K/dual_traverse/dual_traverse_pyccel.py:14-86.
 * stack (stack_cap, 2); m2l, p2p (cap, 2). */
void dual_traverse(const double* t_center, const double* t_half, const i64* t_start,
                   const i64* t_end, const i64* t_child, const double* s_center,
                   const double* s_half, const i64* s_start, const i64* s_end,
                   const i64* s_child, double theta, i64* stack, i64 stack_cap, i64* m2l,
                   i64 m2l_cap, i64* p2p, i64 p2p_cap, i64* counts) {
    double root2 = sqrt(2.0);
    counts[0] = counts[1] = counts[2] = 0;
    stack[0] = 0;
    stack[1] = 0;
    i64 top = 1;
    while (top > 0) {
        top -= 1;
        i64 a = stack[2 * top], b = stack[2 * top + 1];
        if (t_end[a] == t_start[a] || s_end[b] == s_start[b]) continue;
        double dx = t_center[2 * a] - s_center[2 * b];
        double dy = t_center[2 * a + 1] - s_center[2 * b + 1];
        if (root2 * (t_half[a] + s_half[b]) < theta * sqrt(dx * dx + dy * dy)) {
            i64 i = counts[0];
            counts[0] = i + 1;
            if (i < m2l_cap) {
                m2l[2 * i] = a;
                m2l[2 * i + 1] = b;
            } else {
                counts[2] = 1;
            }
            continue;
        }
        int leaf_a = t_child[a] < 0, leaf_b = s_child[b] < 0;
        if (leaf_a && leaf_b) {
            i64 i = counts[1];
            counts[1] = i + 1;
            if (i < p2p_cap) {
                p2p[2 * i] = a;
                p2p[2 * i + 1] = b;
            } else {
                counts[2] = 1;
            }
            continue;
        }
        if (top + 4 > stack_cap) {
            counts[2] = 1;
            return;
        }
        if (leaf_b || (!leaf_a && t_half[a] >= s_half[b])) {
            for (int c = 0; c < 4; ++c) {
                stack[2 * (top + c)] = t_child[a] + c;
                stack[2 * (top + c) + 1] = b;
            }
        } else {
            for (int c = 0; c < 4; ++c) {
                stack[2 * (top + c)] = a;
                stack[2 * (top + c) + 1] = s_child[b] + c;
            }
        }
        top += 4;
    }
}

/* log_targets_host: K/log_targets_host/log_targets_host_pyccel.py:14-94 */
void log_targets_host(const double* tpos, i64 tp_stride, const i64* texclude, i64 t_count,
                      const double* t_center, const i64* t_start, const i64* t_end,
                      const i64* t_child, const double* local_re, const double* local_im,
                      i64 order, const i64* row_start, const i64* partners, const double* spos,
                      i64 sp_stride, const double* scharge, const i64* sindex,
                      const i64* s_start, const i64* s_end, double softening,
                      int with_potential, double* phi, double* field, i64 f_stride) {
    i64 w = order + 1;
    double eps2 = softening * softening;
#pragma omp parallel for schedule(dynamic, 16)
    for (i64 node = 0; node < t_count; ++node) {
        if (t_child[node] >= 0) continue;
        for (i64 k = t_start[node]; k < t_end[node]; ++k) {
            double u_re = tpos[k] - t_center[2 * node];
            double u_im = tpos[tp_stride + k] - t_center[2 * node + 1];
            double w_re = local_re[node * w + order], w_im = local_im[node * w + order];
            double d_re = 0.0, d_im = 0.0;
            for (i64 l = order - 1; l >= 0; --l) {
                double nd_re = d_re * u_re - d_im * u_im + w_re;
                d_im = d_re * u_im + d_im * u_re + w_im;
                d_re = nd_re;
                double nw_re = w_re * u_re - w_im * u_im + local_re[node * w + l];
                w_im = w_re * u_im + w_im * u_re + local_im[node * w + l];
                w_re = nw_re;
            }
            double pot = -2.0 * w_re, ex = 2.0 * d_re, ey = -2.0 * d_im;
            int bad = 0;
            i64 skip = texclude[k];
            for (i64 e = row_start[node]; e < row_start[node + 1]; ++e) {
                i64 src = partners[e];
                for (i64 j = s_start[src]; j < s_end[src]; ++j) {
                    double c = scharge[j];
                    if (c == 0.0 || sindex[j] == skip) continue;
                    double dx = tpos[k] - spos[j], dy = tpos[tp_stride + k] - spos[sp_stride + j];
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad = 1;
                        continue;
                    }
                    if (with_potential) pot -= c * log(r2);
                    ex += 2.0 * c * dx / r2;
                    ey += 2.0 * c * dy / r2;
                }
            }
            if (bad)
                phi[k] = 1.0e300;
            else if (with_potential)
                phi[k] = pot;
            else
                phi[k] = 0.0;
            field[k] = ex;
            field[f_stride + k] = ey;
        }
    }
}

/* cart_targets_host: K/cart_targets_host/cart_targets_host_pyccel.py:16-98 */
void cart_targets_host(const double* tpos, i64 tp_stride, const i64* texclude, i64 t_count,
                       const double* t_center, const i64* t_start, const i64* t_end,
                       const i64* t_child, const double* local, i64 n_coef,
                       const i64* mono_parent, const i64* mono_dir, const i64* ex_pow,
                       const i64* ey_pow, const i64* grad, const i64* row_start,
                       const i64* partners, const double* spos, i64 sp_stride,
                       const double* scharge, const i64* sindex, const i64* s_start,
                       const i64* s_end, double softening, double* phi, double* field,
                       i64 f_stride) {
    double eps2 = softening * softening;
#pragma omp parallel for schedule(dynamic, 16)
    for (i64 node = 0; node < t_count; ++node) {
        double mono[2145];
        if (t_child[node] >= 0) continue;
        const double* L = local + node * n_coef;
        for (i64 k = t_start[node]; k < t_end[node]; ++k) {
            mono[0] = 1.0;
            for (i64 i = 1; i < n_coef; ++i) {
                if (mono_dir[i] == 0)
                    mono[i] = mono[mono_parent[i]] * (tpos[k] - t_center[2 * node]);
                else
                    mono[i] = mono[mono_parent[i]] * (tpos[tp_stride + k] - t_center[2 * node + 1]);
            }
            double pot = 0.0, ex = 0.0, ey = 0.0;
            for (i64 i = 0; i < n_coef; ++i) {
                pot += L[i] * mono[i];
                if (grad[2 * i] >= 0) ex -= (double)ex_pow[i] * L[i] * mono[grad[2 * i]];
                if (grad[2 * i + 1] >= 0) ey -= (double)ey_pow[i] * L[i] * mono[grad[2 * i + 1]];
            }
            int bad = 0;
            i64 skip = texclude[k];
            for (i64 e = row_start[node]; e < row_start[node + 1]; ++e) {
                i64 src = partners[e];
                for (i64 j = s_start[src]; j < s_end[src]; ++j) {
                    double c = scharge[j];
                    if (c == 0.0 || sindex[j] == skip) continue;
                    double dx = tpos[k] - spos[j], dy = tpos[tp_stride + k] - spos[sp_stride + j];
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad = 1;
                        continue;
                    }
                    double inv_r = 1.0 / sqrt(r2);
                    double inv_r3 = inv_r * inv_r * inv_r;
                    pot += c * inv_r;
                    ex += c * inv_r3 * dx;
                    ey += c * inv_r3 * dy;
                }
            }
            phi[k] = bad ? 1.0e300 : pot;
            field[k] = ex;
            field[f_stride + k] = ey;
        }
    }
}
