/*
 * Mesh construction on the host, once per case.
 *
 * ccfd_mesh_build() produces the connectivity and geometry of createMesh
 * (src/mesh.c:1405-1844) in flat arrays, in the reference's own element,
 * face and half-side order and with the same floating-point expressions, so
 * that the geometry is bit-identical to the reference's:
 *   - elements: triangles then quadrilaterals (src/mesh.c:1493-1647); each
 *     element's half-sides are created for node pairs (k, k+1) and prepended
 *     to its side list, so the list runs in reverse creation order
 *     (src/mesh.c:1548-1549, 1625-1626);
 *   - faces: half-sides sorted by (min node, max node, is-boundary) and paired
 *     (src/mesh.c:1710-1755); the first of a pair owns the face (boundary
 *     pairs: the physical side), faces are prepended to the face list and
 *     boundary ghosts to the BC list.  The sort is a stable merge sort, the
 *     behaviour of glibc's qsort on which the reference relies for the
 *     owner of interior faces;
 *   - geometry: createElemInfo (src/mesh.c:296-341), createSideInfo
 *     (src/mesh.c:250-289, ghost barycentre mirrored across the face),
 *     createReconstructionInfo (src/mesh.c:80-114, least-squares weights from
 *     a Gram-Schmidt factorisation of the barycentre-to-barycentre vectors).
 *   - periodic boundaries: connectPeriodicBC (src/mesh.c:172-244) joins the
 *     matched boundary faces into interior faces before the least-squares
 *     weights are formed.
 *
 * Also here: the Cartesian generator (src/mesh.c:385-486), the gmsh 2.2,
 * gmsh 4 and EMC2 readers (src/mesh.c:498-1139) and a gmsh 2.2 writer.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ccfd_host.h"

typedef struct hside {
	long node[2];     /* node ids as created                          */
	long key0, key1;  /* min / max node id                            */
	int is_bc;        /* boundary edge                                */
	long elem;        /* owning cell, or -1 for a ghost side          */
	int bc;           /* BC table index of a ghost side (-1 if none)  */
	long conn;        /* paired half-side                             */
	long ghost;       /* ghost index (BCside order) of a ghost side   */
	double gp[2], n[2], len, bb[2], bbd, w[2];
} hside;

static int key_less(const hside *hs, long a, long b)
{
	/* compare() of src/mesh.c:362-375 */
	if (hs[a].key0 != hs[b].key0)
		return hs[a].key0 < hs[b].key0;
	if (hs[a].key1 != hs[b].key1)
		return hs[a].key1 < hs[b].key1;
	return hs[a].is_bc < hs[b].is_bc;
}

/* stable bottom-up merge sort of half-side indices */
static int stable_sort(const hside *hs, long *idx, long n)
{
	long *tmp = malloc(sizeof(long) * (n > 0 ? n : 1));
	if (!tmp)
		return CCFD_ERR_NOMEM;
	for (long width = 1; width < n; width *= 2) {
		for (long lo = 0; lo < n; lo += 2 * width) {
			long mid = lo + width < n ? lo + width : n;
			long hi = lo + 2 * width < n ? lo + 2 * width : n;
			long i = lo, j = mid, k = lo;
			while (i < mid && j < hi) {
				if (key_less(hs, idx[j], idx[i]))
					tmp[k++] = idx[j++];
				else
					tmp[k++] = idx[i++];
			}
			while (i < mid)
				tmp[k++] = idx[i++];
			while (j < hi)
				tmp[k++] = idx[j++];
		}
		memcpy(idx, tmp, sizeof(long) * n);
	}
	free(tmp);
	return CCFD_OK;
}

void ccfd_mesh_free(ccfd_mesh *m)
{
	if (!m)
		return;
	free(m->cell_type); free(m->cell_domain); free(m->cell_bary);
	free(m->cell_geo); free(m->hs_offset); free(m->hs_face);
	free(m->hs_sign); free(m->hs_nb); free(m->hs_gp); free(m->hs_w);
	free(m->face_cells); free(m->face_hs); free(m->face_n);
	free(m->face_len); free(m->face_bb); free(m->ghost_gp);
	free(m->bc_face); free(m->bc_index); free(m->bc_ghost_bary);
	free(m->bc_x);
	free(m->cell_gp5);
	free(m->cell_nodes);
	free(m->node_xy);
	memset(m, 0, sizeof(*m));
}

static int find_bc(const ccfd_bc *tab, int n, int code)
{
	/* the reference prepends BCs (src/boundary.c:44-45) and takes the first
	 * match in list order: the last one defined */
	int type = code / 100, id = code % 100;
	for (int i = n - 1; i >= 0; --i)
		if (tab[i].type == type && tab[i].id == id)
			return i;
	return -1;
}

int ccfd_mesh_build(const double *nodes, long n_nodes,
		    const long *tria, long n_tria, const long *quad, long n_quad,
		    const long *bc_edge, long n_bc_edge,
		    const ccfd_bc *bc_table, int n_bc_table, ccfd_mesh *m)
{
	memset(m, 0, sizeof(*m));
	if (n_nodes <= 0 || n_tria + n_quad <= 0)
		return CCFD_ERR_MESH;
	long n_elem = n_tria + n_quad;
	long n_created = 3 * n_tria + 4 * n_quad + n_bc_edge;
	if (n_created % 2)
		return CCFD_ERR_MESH;
	long n_sides = n_created / 2;

	hside *hs = calloc(n_created, sizeof(hside));
	long *elem_first = malloc(sizeof(long) * n_elem);
	int *etype = malloc(sizeof(int) * n_elem);
	int *edom = malloc(sizeof(int) * n_elem);
	long *enode = malloc(sizeof(long) * 4 * n_elem);
	double *bary = malloc(sizeof(double) * 2 * n_elem);
	double *geo = malloc(sizeof(double) * 4 * n_elem);
	long *idx = malloc(sizeof(long) * n_created);
	long *pair_a = malloc(sizeof(long) * n_sides);
	long *pair_b = malloc(sizeof(long) * n_sides);
	if (!hs || !elem_first || !etype || !edom || !enode || !bary || !geo ||
	    !idx || !pair_a || !pair_b) {
		free(hs); free(elem_first); free(etype); free(edom); free(enode);
		free(bary); free(geo); free(idx); free(pair_a); free(pair_b);
		return CCFD_ERR_NOMEM;
	}
	int st = CCFD_OK;

	/* x/y extents over all nodes (src/mesh.c:1465-1488) */
	m->x_min = m->x_max = nodes[0];
	m->y_min = m->y_max = nodes[1];
	for (long i = n_nodes - 1; i >= 0; --i) {
		m->x_min = fmin(nodes[2 * i], m->x_min);
		m->x_max = fmax(nodes[2 * i], m->x_max);
		m->y_min = fmin(nodes[2 * i + 1], m->y_min);
		m->y_max = fmax(nodes[2 * i + 1], m->y_max);
	}

	/* elements and their half-sides in creation order */
	long ns = 0;
	for (long e = 0; e < n_elem; ++e) {
		int t = e < n_tria ? 3 : 4;
		const long *src = e < n_tria ? &tria[4 * e] : &quad[5 * (e - n_tria)];
		etype[e] = t;
		edom[e] = (int)src[t];
		for (int k = 0; k < t; ++k) {
			if (src[k] < 0 || src[k] >= n_nodes) {
				st = CCFD_ERR_MESH;
				goto done;
			}
			enode[4 * e + k] = src[k];
		}
		double bx = 0.0, by = 0.0;
		for (int k = 0; k < t; ++k) {
			bx += nodes[2 * enode[4 * e + k]] / t;
			by += nodes[2 * enode[4 * e + k] + 1] / t;
		}
		bary[2 * e] = bx;
		bary[2 * e + 1] = by;
		elem_first[e] = ns;
		for (int k = 0; k < t; ++k, ++ns) {
			long a = enode[4 * e + k], b = enode[4 * e + (k + 1) % t];
			hs[ns].node[0] = a;
			hs[ns].node[1] = b;
			hs[ns].key0 = a < b ? a : b;
			hs[ns].key1 = a < b ? b : a;
			hs[ns].is_bc = 0;
			hs[ns].elem = e;
			hs[ns].bc = -1;
			hs[ns].ghost = -1;
		}
	}
	for (long k = 0; k < n_bc_edge; ++k, ++ns) {
		long a = bc_edge[3 * k], b = bc_edge[3 * k + 1];
		if (a < 0 || a >= n_nodes || b < 0 || b >= n_nodes) {
			st = CCFD_ERR_MESH;
			goto done;
		}
		int code = (int)bc_edge[3 * k + 2];
		int bi = find_bc(bc_table, n_bc_table, code);
		if (bi < 0 || code / 100 == 0) {
			st = CCFD_ERR_MESH; /* BC missing from the parameter file */
			goto done;
		}
		hs[ns].node[0] = a;
		hs[ns].node[1] = b;
		hs[ns].key0 = a < b ? a : b;
		hs[ns].key1 = a < b ? b : a;
		hs[ns].is_bc = 1;
		hs[ns].elem = -1;
		hs[ns].bc = bi;
		hs[ns].ghost = -1;
	}

	/* pair half-sides into faces (src/mesh.c:1710-1755) */
	for (long i = 0; i < n_created; ++i)
		idx[i] = i;
	if ((st = stable_sort(hs, idx, n_created)) != CCFD_OK)
		goto done;
	long n_ghost = 0;
	for (long p = 0; p < n_sides; ++p) {
		long a = idx[2 * p], b = idx[2 * p + 1];
		if (hs[a].key0 != hs[b].key0 || hs[a].key1 != hs[b].key1 ||
		    (hs[a].is_bc && hs[b].is_bc)) {
			st = CCFD_ERR_MESH; /* "Problem in Connect" */
			goto done;
		}
		if (hs[a].is_bc) {
			long c = a; a = b; b = c;
		}
		pair_a[p] = a;
		pair_b[p] = b;
		hs[a].conn = b;
		hs[b].conn = a;
		if (hs[b].is_bc)
			++n_ghost;
	}

	/* ghosts in BCside order: the reverse of the pairing order */
	{
		long g = n_ghost;
		for (long p = 0; p < n_sides; ++p)
			if (hs[pair_b[p]].is_bc)
				hs[pair_b[p]].ghost = --g;
	}

	/* createElemInfo, element order (src/mesh.c:296-341) */
	double total_area_q = 0.0;
	for (long e = 0; e < n_elem; ++e) {
		int t = etype[e];
		double bx = 0.0, by = 0.0;
		for (int k = 0; k < t; ++k) {
			bx += nodes[2 * enode[4 * e + k]] / t;
			by += nodes[2 * enode[4 * e + k] + 1] / t;
		}
		bary[2 * e] = bx;
		bary[2 * e + 1] = by;
		double nn[4][2] = {{0}}, len[4] = {0};
		for (int i = 0; i < t; ++i) {
			int j = (i + 1) % t;
			const double *xi = &nodes[2 * enode[4 * e + i]];
			const double *xj = &nodes[2 * enode[4 * e + j]];
			double vx = xj[0] - xi[0], vy = xj[1] - xi[1];
			len[i] = sqrt(vx * vx + vy * vy);
			nn[i][0] = xj[1] - xi[1];
			nn[i][1] = xi[0] - xj[0];
			double tmp = sqrt(nn[i][0] * nn[i][0] + nn[i][1] * nn[i][1]);
			nn[i][0] /= tmp;
			nn[i][1] /= tmp;
		}
		double area = 0.5 * len[0] * len[1] *
			fabs(nn[0][0] * nn[1][1] - nn[1][0] * nn[0][1]);
		if (t == 4)
			area += 0.5 * len[2] * len[3] *
				fabs(nn[2][0] * nn[3][1] - nn[3][0] * nn[2][1]);
		double areaq = 1.0 / area;
		if (total_area_q != 0.0)
			total_area_q = 1.0 / (1.0 / total_area_q + area);
		else
			total_area_q = areaq;
		double sx = 0, sy = 0;
		for (int i = 0; i < t; ++i) {
			sx += fabs(nn[i][0]) * len[i] / 2.0;
			sy += fabs(nn[i][1]) * len[i] / 2.0;
		}
		geo[4 * e + 0] = area;
		geo[4 * e + 1] = areaq;
		geo[4 * e + 2] = sx;
		geo[4 * e + 3] = sy;
	}

	/* createSideInfo per face (src/mesh.c:250-289) */
	double *ghost_bary = malloc(sizeof(double) * 2 * (n_ghost + 1));
	if (!ghost_bary) {
		st = CCFD_ERR_NOMEM;
		goto done;
	}
	for (long p = 0; p < n_sides; ++p) {
		hside *A = &hs[pair_a[p]], *B = &hs[pair_b[p]];
		const double *x0 = &nodes[2 * A->node[0]], *x1 = &nodes[2 * A->node[1]];
		double nx = x1[1] - x0[1];
		double ny = x0[0] - x1[0];
		double len = sqrt(nx * nx + ny * ny);
		nx /= len;
		ny /= len;
		double gx = 0.5 * (x0[0] + x1[0]);
		double gy = 0.5 * (x0[1] + x1[1]);
		A->gp[0] = gx - bary[2 * A->elem];
		A->gp[1] = gy - bary[2 * A->elem + 1];
		if ((nx * A->gp[0] + ny * A->gp[1]) < 0.0) {
			nx *= -1.0;
			ny *= -1.0;
		}
		A->n[0] = nx;
		A->n[1] = ny;
		A->len = len;
		double cbx, cby;
		if (B->is_bc) {
			double tmp = 2.0 * fabs(A->gp[0] * nx + A->gp[1] * ny);
			cbx = bary[2 * A->elem] + tmp * nx;
			cby = bary[2 * A->elem + 1] + tmp * ny;
			ghost_bary[2 * B->ghost] = cbx;
			ghost_bary[2 * B->ghost + 1] = cby;
		} else {
			cbx = bary[2 * B->elem];
			cby = bary[2 * B->elem + 1];
		}
		B->gp[0] = gx - cbx;
		B->gp[1] = gy - cby;
		B->n[0] = -nx;
		B->n[1] = -ny;
		B->len = len;
	}

	/* connectPeriodicBC (src/mesh.c:172-244): in BC-list order, the ghost of
	 * a periodic BC whose id ends in 1 is matched with the first ghost of
	 * the periodic BC with the same id / 10 and an id ending in 2 whose face
	 * midpoint is its own plus the BC's connection vector (within 1e-7 in
	 * the 1-norm).  The two interior half-sides then face each other across
	 * one interior face, owned by the first; the second one's face and both
	 * ghosts leave the face and BC lists (src/mesh.c:1834-1841). */
	long *gpair = malloc(sizeof(long) * (n_ghost + 1));  /* ghost -> face pair */
	long *gside = malloc(sizeof(long) * (n_ghost + 1));  /* ghost -> its half-side */
	long *gnew = malloc(sizeof(long) * (n_ghost + 1));   /* ghost -> BC-list index or -1 */
	char *removed = calloc(n_sides + 1, 1);
	char *matched = calloc(n_ghost + 1, 1);
	long *face_new = malloc(sizeof(long) * (n_sides + 1));
	if (!gpair || !gside || !gnew || !removed || !matched || !face_new) {
		free(gpair); free(gside); free(gnew); free(removed); free(matched); free(face_new);
		free(ghost_bary);
		st = CCFD_ERR_NOMEM;
		goto done;
	}
	for (long p = 0; p < n_sides; ++p)
		if (hs[pair_b[p]].is_bc) {
			gpair[hs[pair_b[p]].ghost] = p;
			gside[hs[pair_b[p]].ghost] = pair_b[p];
		}
	for (long g = 0; g < n_ghost && st == CCFD_OK; ++g) {
		const hside *G = &hs[gside[g]];
		const ccfd_bc *bc = &bc_table[G->bc];
		if (bc->type != CCFD_BC_PERIODIC || bc->id % 10 != 1)
			continue;
		double ax = G->gp[0] + ghost_bary[2 * g], ay = G->gp[1] + ghost_bary[2 * g + 1];
		long hit = -1;
		for (long g2 = 0; g2 < n_ghost && hit < 0; ++g2) {
			const hside *S = &hs[gside[g2]];
			const ccfd_bc *sb = &bc_table[S->bc];
			if (sb->type != CCFD_BC_PERIODIC || sb->id % 10 != 2 || sb->id / 10 != bc->id / 10)
				continue;
			double sx = S->gp[0] + ghost_bary[2 * g2], sy = S->gp[1] + ghost_bary[2 * g2 + 1];
			if ((fabs(ax + bc->connection[0] - sx) + fabs(ay + bc->connection[1] - sy)) <= 1e-7)
				hit = g2;
		}
		if (hit < 0) {
			st = CCFD_ERR_MESH; /* "No connection found" */
			break;
		}
		long p = gpair[g], p2 = gpair[hit];
		long ur = pair_a[p], target = pair_a[p2];
		hs[ur].conn = target;
		hs[target].conn = ur;
		pair_b[p] = target;
		removed[p2] = 1;
		matched[hit] = 1;
	}
	/* a periodic ghost with an id ending in 2 that no ghost connected would
	 * stay a ghost whose state is never set: rejected */
	for (long g = 0; g < n_ghost && st == CCFD_OK; ++g) {
		const ccfd_bc *bc = &bc_table[hs[gside[g]].bc];
		if (bc->type == CCFD_BC_PERIODIC && bc->id % 10 != 1 && !matched[g])
			st = CCFD_ERR_MESH;
	}
	if (st == CCFD_OK) {
		long gn = 0;
		for (long g = 0; g < n_ghost; ++g)
			gnew[g] = bc_table[hs[gside[g]].bc].type == CCFD_BC_PERIODIC ? -1 : gn++;
		long fn = 0;
		for (long p = n_sides - 1; p >= 0; --p)  /* face list order */
			face_new[p] = removed[p] ? -1 : fn++;
	}
	free(gpair);
	free(gside);
	free(matched);
	if (st != CCFD_OK) {
		free(gnew); free(removed); free(face_new); free(ghost_bary);
		goto done;
	}

	/* createReconstructionInfo per element (src/mesh.c:80-114) */
	for (long e = 0; e < n_elem; ++e) {
		int t = etype[e];
		double r11 = 0.0, r12 = 0.0, r22 = 0.0;
		for (int k = t - 1; k >= 0; --k) {
			hside *S = &hs[elem_first[e] + k];
			hside *C = &hs[S->conn];
			S->bb[0] = S->gp[0] - C->gp[0];
			S->bb[1] = S->gp[1] - C->gp[1];
			S->bbd = sqrt(S->bb[0] * S->bb[0] + S->bb[1] * S->bb[1]);
			r11 += S->bb[0] * S->bb[0];
			r12 += S->bb[0] * S->bb[1];
			r22 += S->bb[1] * S->bb[1];
		}
		r11 = sqrt(r11);
		r12 = r12 / r11;
		r22 = sqrt(r22 - r12 * r12);
		for (int k = t - 1; k >= 0; --k) {
			hside *S = &hs[elem_first[e] + k];
			double alpha1 = S->bb[0] / (r11 * r11);
			double alpha2 = (S->bb[1] - r12 / r11 * S->bb[0]) / (r22 * r22);
			S->w[0] = alpha1 - r12 / r11 * alpha2;
			S->w[1] = alpha2;
		}
	}

	/* flatten, faces in side[] order = reverse pairing order */
	long F = 0, N = n_elem, H = 3 * n_tria + 4 * n_quad, B = 0;
	for (long p = 0; p < n_sides; ++p)
		F += !removed[p];
	for (long g = 0; g < n_ghost; ++g)
		B += gnew[g] >= 0;
	m->n_cells = N;
	m->n_faces = F;
	m->n_bc = B;
	m->n_half_sides = H;
	m->n_nodes = n_nodes;
	m->cell_type = malloc(sizeof(int) * N);
	m->cell_domain = malloc(sizeof(int) * N);
	m->cell_bary = malloc(sizeof(double) * 2 * N);
	m->cell_gp5 = malloc(sizeof(double) * 2 * N);
	m->cell_nodes = malloc(sizeof(long) * 4 * N);
	m->node_xy = malloc(sizeof(double) * 2 * n_nodes);
	m->cell_geo = malloc(sizeof(double) * 4 * N);
	m->hs_offset = malloc(sizeof(long) * (N + 1));
	m->hs_face = malloc(sizeof(long) * H);
	m->hs_sign = malloc(sizeof(int) * H);
	m->hs_nb = malloc(sizeof(long) * H);
	m->hs_gp = malloc(sizeof(double) * 2 * H);
	m->hs_w = malloc(sizeof(double) * 2 * H);
	m->face_cells = malloc(sizeof(long) * 2 * F);
	m->face_hs = malloc(sizeof(long) * 2 * F);
	m->face_n = malloc(sizeof(double) * 2 * F);
	m->face_len = malloc(sizeof(double) * F);
	m->face_bb = malloc(sizeof(double) * 3 * F);
	m->ghost_gp = malloc(sizeof(double) * 2 * (B + 1));
	m->bc_face = malloc(sizeof(long) * (B + 1));
	m->bc_index = malloc(sizeof(int) * (B + 1));
	m->bc_ghost_bary = malloc(sizeof(double) * 2 * (B + 1));
	m->bc_x = malloc(sizeof(double) * 2 * (B + 1));
	long *hs_face_of = malloc(sizeof(long) * n_created);
	long *hs_pos = malloc(sizeof(long) * n_created);
	if (!m->cell_type || !m->cell_domain || !m->cell_bary || !m->cell_geo || !m->cell_gp5 ||
	    !m->cell_nodes || !m->node_xy ||
	    !m->hs_offset || !m->hs_face || !m->hs_sign || !m->hs_nb ||
	    !m->hs_gp || !m->hs_w || !m->face_cells || !m->face_hs ||
	    !m->face_n || !m->face_len || !m->face_bb || !m->ghost_gp ||
	    !m->bc_face || !m->bc_index || !m->bc_ghost_bary || !m->bc_x ||
	    !hs_face_of || !hs_pos) {
		free(hs_face_of); free(hs_pos); free(ghost_bary);
		free(gnew); free(removed); free(face_new);
		ccfd_mesh_free(m);
		st = CCFD_ERR_NOMEM;
		goto done;
	}
	for (long p = 0; p < n_sides; ++p) {
		if (removed[p])
			continue;
		hs_face_of[pair_a[p]] = face_new[p];
		hs_face_of[pair_b[p]] = face_new[p];
	}
	long k = 0;
	for (long e = 0; e < N; ++e) {
		m->cell_type[e] = etype[e];
		m->cell_domain[e] = edom[e];
		m->cell_bary[2 * e] = bary[2 * e];
		m->cell_bary[2 * e + 1] = bary[2 * e + 1];
		if (etype[e] == 4) {
			const double *x0 = &nodes[2 * enode[4 * e]], *x2 = &nodes[2 * enode[4 * e + 2]];
			m->cell_gp5[2 * e] = 0.5 * (x0[0] + x2[0]);
			m->cell_gp5[2 * e + 1] = 0.5 * (x0[1] + x2[1]);
		} else {
			m->cell_gp5[2 * e] = bary[2 * e];
			m->cell_gp5[2 * e + 1] = bary[2 * e + 1];
		}
		memcpy(&m->cell_geo[4 * e], &geo[4 * e], sizeof(double) * 4);
		for (int j = 0; j < 4; ++j)
			m->cell_nodes[4 * e + j] = j < etype[e] ? enode[4 * e + j] : -1;
		m->hs_offset[e] = k;
		for (int j = etype[e] - 1; j >= 0; --j, ++k) {
			long s = elem_first[e] + j;
			hside *S = &hs[s], *C = &hs[S->conn];
			hs_pos[s] = k;
			m->hs_face[k] = hs_face_of[s];
			m->hs_sign[k] = 0;
			m->hs_nb[k] = C->is_bc ? -1 - gnew[C->ghost] : C->elem;
			m->hs_gp[2 * k] = S->gp[0];
			m->hs_gp[2 * k + 1] = S->gp[1];
			m->hs_w[2 * k] = S->w[0];
			m->hs_w[2 * k + 1] = S->w[1];
		}
	}
	m->hs_offset[N] = k;
	for (long p = 0; p < n_sides; ++p) {
		if (removed[p])
			continue;
		long f = face_new[p];
		hside *A = &hs[pair_a[p]], *Bs = &hs[pair_b[p]];
		m->hs_sign[hs_pos[pair_a[p]]] = 1;
		m->face_cells[2 * f] = A->elem;
		m->face_hs[2 * f] = hs_pos[pair_a[p]];
		if (Bs->is_bc) {
			long g = gnew[Bs->ghost];
			m->face_cells[2 * f + 1] = -1 - g;
			m->face_hs[2 * f + 1] = -1;
			m->bc_face[g] = f;
			m->bc_index[g] = Bs->bc;
			m->bc_ghost_bary[2 * g] = ghost_bary[2 * Bs->ghost];
			m->bc_ghost_bary[2 * g + 1] = ghost_bary[2 * Bs->ghost + 1];
			m->ghost_gp[2 * g] = Bs->gp[0];
			m->ghost_gp[2 * g + 1] = Bs->gp[1];
			m->bc_x[2 * g] = A->gp[0] + bary[2 * A->elem];
			m->bc_x[2 * g + 1] = A->gp[1] + bary[2 * A->elem + 1];
		} else {
			m->hs_sign[hs_pos[pair_b[p]]] = -1;
			m->face_cells[2 * f + 1] = Bs->elem;
			m->face_hs[2 * f + 1] = hs_pos[pair_b[p]];
		}
		m->face_n[2 * f] = A->n[0];
		m->face_n[2 * f + 1] = A->n[1];
		m->face_len[f] = A->len;
		m->face_bb[3 * f] = A->bb[0];
		m->face_bb[3 * f + 1] = A->bb[1];
		m->face_bb[3 * f + 2] = A->bbd;
	}
	memcpy(m->node_xy, nodes, sizeof(double) * 2 * n_nodes);
	m->total_area_q = total_area_q;
	m->dx_ref = sqrt(1.0 / (total_area_q * N));
	free(hs_face_of);
	free(hs_pos);
	free(ghost_bary);
	free(gnew);
	free(removed);
	free(face_new);
done:
	free(hs); free(elem_first); free(etype); free(edom); free(enode);
	free(bary); free(geo); free(idx); free(pair_a); free(pair_b);
	return st;
}

void ccfd_venk_eps2(const ccfd_mesh *m, double venk_k, double *eps2)
{
	/* src/finiteVolume.c:47-52 */
	for (long e = 0; e < m->n_cells; ++e) {
		double area = m->cell_geo[4 * e];
		eps2[e] = (venk_k * sqrt(area)) * (venk_k * sqrt(area)) *
			  (venk_k * sqrt(area));
	}
}

int ccfd_locate_points(const ccfd_mesh *m, const double *xy, int n, long *cells_out)
{
	if (!m || (n > 0 && (!xy || !cells_out)) || !m->cell_nodes || !m->node_xy)
		return CCFD_ERR_ARG;
	/* initRecordPoints, src/analyze.c:43-82.  The edge normal is divided by
	 * sqrt(2 u_x^2) as there (u_y does not enter); for an edge with u_x = 0
	 * the projection is not a number and the edge excludes nothing. */
	for (int p = 0; p < n; ++p) {
		const double *pt = &xy[2 * p];
		long found = -1;
		for (long e = 0; e < m->n_cells && found < 0; ++e) {
			int t = m->cell_type[e];
			int inside = 1;
			for (int i = 0; i < t; ++i) {
				int j = i + 1 < t ? i + 1 : 0;
				const double *x1 = &m->node_xy[2 * m->cell_nodes[4 * e + i]];
				const double *x2 = &m->node_xy[2 * m->cell_nodes[4 * e + j]];
				double u[2] = {x2[1] - x1[1], x1[0] - x2[0]};
				double tmp = sqrt(u[0] * u[0] + u[0] * u[0]);
				u[0] /= tmp;
				u[1] /= tmp;
				double x[2] = {pt[0] - x1[0], pt[1] - x1[1]};
				double projection = u[0] * x[0] + u[1] * x[1];
				if (projection > 0.0)
					inside = 0;
			}
			if (inside)
				found = e;
		}
		if (found < 0)
			return CCFD_ERR_MESH; /* "Record Point # is not in Domain" */
		cells_out[p] = found;
	}
	return CCFD_OK;
}

/* ------------------------------------------------------------ Cartesian */
int ccfd_cart_generate(const ccfd_cart *c, double **nodes_out, long *n_nodes,
		       long **quad_out, long *n_quad, long **bc_out, long *n_bc)
{
	long iMax = c->i_max, jMax = c->j_max;
	if (iMax <= 0 || jMax <= 0)
		return CCFD_ERR_MESH;
	long nv = (iMax + 1) * (jMax + 1), nq = iMax * jMax;
	long nb = 0;
	for (int s = 0; s < 4; ++s)
		for (int b = 0; b < c->n_bc[s]; ++b)
			nb += c->bc_range[s][b][1] - c->bc_range[s][b][0] + 1;
	double *nodes = malloc(sizeof(double) * 2 * nv);
	long *quad = malloc(sizeof(long) * 5 * nq);
	long *bc = malloc(sizeof(long) * 3 * (nb + 1));
	if (!nodes || !quad || !bc) {
		free(nodes); free(quad); free(bc);
		return CCFD_ERR_NOMEM;
	}
	double dx = (c->x_max - c->x_min) / iMax;
	double dy = (c->y_max - c->y_min) / jMax;
	double y = c->y_min, x;
	long k = 0;
	for (long j = 0; j < jMax + 1; ++j) {
		x = c->x_min;
		for (long i = 0; i < iMax + 1; ++i) {
			nodes[2 * k] = x;
			nodes[2 * k + 1] = y;
			k++;
			x += dx;
		}
		y += dy;
	}
	k = 0;
	for (long j = 0; j < jMax; ++j)
		for (long i = 0; i < iMax; ++i) {
			quad[5 * k + 0] = k + j;
			quad[5 * k + 1] = k + j + 1;
			quad[5 * k + 2] = k + j + 1 + iMax + 1;
			quad[5 * k + 3] = k + j + iMax + 1;
			quad[5 * k + 4] = 1;
			k++;
		}
	k = 0;
	for (int s = 0; s < 4; ++s)
		for (int b = 0; b < c->n_bc[s]; ++b)
			for (long i = c->bc_range[s][b][0] - 1; i < c->bc_range[s][b][1]; ++i) {
				long a0, a1;
				switch (s) {
				case 0: a0 = i; a1 = i + 1; break;
				case 1: a0 = (iMax + 1) * (i + 1) - 1; a1 = (iMax + 1) * (i + 2) - 1; break;
				case 2: a0 = (iMax + 1) * jMax + i; a1 = a0 + 1; break;
				default: a0 = i * (iMax + 1); a1 = a0 + iMax + 1; break;
				}
				bc[3 * k] = a0;
				bc[3 * k + 1] = a1;
				bc[3 * k + 2] = c->bc_type[s][b];
				k++;
			}
	*nodes_out = nodes;
	*n_nodes = nv;
	*quad_out = quad;
	*n_quad = nq;
	*bc_out = bc;
	*n_bc = nb;
	return CCFD_OK;
}

/* ------------------------------------------------------------ gmsh 2.2 */
int ccfd_write_gmsh2(const char *path, const double *nodes, long n_nodes,
		     const long *tria, long n_tria, const long *quad, long n_quad,
		     const long *bc_edge, long n_bc_edge)
{
	FILE *f = fopen(path, "w");
	if (!f)
		return CCFD_ERR_ARG;
	fprintf(f, "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%ld\n", n_nodes);
	for (long i = 0; i < n_nodes; ++i)
		fprintf(f, "%ld %.17g %.17g 0\n", i + 1, nodes[2 * i], nodes[2 * i + 1]);
	fprintf(f, "$EndNodes\n$Elements\n%ld\n", n_bc_edge + n_tria + n_quad);
	long id = 1;
	for (long i = 0; i < n_bc_edge; ++i)
		fprintf(f, "%ld 1 2 %ld %ld %ld %ld\n", id++, bc_edge[3 * i + 2],
			bc_edge[3 * i + 2], bc_edge[3 * i] + 1, bc_edge[3 * i + 1] + 1);
	for (long i = 0; i < n_tria; ++i)
		fprintf(f, "%ld 2 2 %ld %ld %ld %ld %ld\n", id++, tria[4 * i + 3],
			tria[4 * i + 3], tria[4 * i] + 1, tria[4 * i + 1] + 1,
			tria[4 * i + 2] + 1);
	for (long i = 0; i < n_quad; ++i)
		fprintf(f, "%ld 3 2 %ld %ld %ld %ld %ld %ld\n", id++, quad[5 * i + 4],
			quad[5 * i + 4], quad[5 * i] + 1, quad[5 * i + 1] + 1,
			quad[5 * i + 2] + 1, quad[5 * i + 3] + 1);
	fprintf(f, "$EndElements\n");
	int err = ferror(f);
	fclose(f);
	return err ? CCFD_ERR_ARG : CCFD_OK;
}

/* gmsh 2.x ASCII reader with the rules of readGmsh (src/mesh.c:528-742):
 * line elements whose first tag (physical group) is > 100 are BC edges with
 * that code, triangles / quads carry their physical group as the domain;
 * other elements are ignored.  gmsh 4 files are not read. */
/* gmsh 4 as the reference reads it (readGmsh, src/mesh.c:743-983): the
 * physical tag of every curve entity that has one, in $Entities order;
 * nodes by entity blocks (tags must run 1..n); element blocks of lines
 * (boundary edges whose BC code is the physical tag at the block's own
 * index), triangles and quadrilaterals (domain 1); lines of blocks of other
 * element types are not consumed, as there. */
static int read_gmsh4(FILE *f, double **nodes_out, long *n_nodes, long **tria_out, long *n_tria,
		      long **quad_out, long *n_quad, long **bc_out, long *n_bc)
{
	char line[8192];
	long np = -1, nc = 0;
	int st = CCFD_OK;
	int *ptag = NULL;
	long nptag = 0, nv = 0, ne = 0, nb = 0, nt = 0, nq = 0;
	double *nodes = NULL;
	long *tria = NULL, *quad = NULL, *bc = NULL;
	rewind(f);
	while (fgets(line, sizeof(line), f))
		if (!strcmp(line, "$Entities\n")) {
			if (!fgets(line, sizeof(line), f) || sscanf(line, "%ld %ld", &np, &nc) != 2)
				return CCFD_ERR_MESH;
			break;
		}
	if (np < 0 || nc <= 0)
		return CCFD_ERR_MESH; /* "No curves in mesh file" */
	ptag = malloc(sizeof(int) * nc);
	if (!ptag)
		return CCFD_ERR_NOMEM;
	for (long l = 0; l < np; ++l)
		if (!fgets(line, sizeof(line), f)) {
			st = CCFD_ERR_MESH;
			goto out;
		}
	for (long l = 0; l < nc; ++l) {
		if (!fgets(line, sizeof(line), f)) {
			st = CCFD_ERR_MESH;
			goto out;
		}
		char *save = NULL, *tok = strtok_r(line, " ", &save);
		for (int k = 0; k < 7 && tok; ++k)
			tok = strtok_r(NULL, " ", &save);
		if (!tok) {
			st = CCFD_ERR_MESH;
			goto out;
		}
		if (strtol(tok, NULL, 10)) {
			tok = strtok_r(NULL, " ", &save);
			if (!tok) {
				st = CCFD_ERR_MESH;
				goto out;
			}
			ptag[nptag++] = (int)strtol(tok, NULL, 10);
		}
	}
	int nblk = 0;
	rewind(f);
	while (fgets(line, sizeof(line), f))
		if (!strcmp(line, "$Nodes\n")) {
			if (!fgets(line, sizeof(line), f) || sscanf(line, "%d %ld", &nblk, &nv) != 2)
				nv = 0;
			break;
		}
	if (nv <= 0) {
		st = CCFD_ERR_MESH; /* "No Nodes in Mesh file" */
		goto out;
	}
	nodes = malloc(sizeof(double) * 2 * nv);
	long *ids = malloc(sizeof(long) * nv);
	if (!nodes || !ids) {
		free(ids);
		st = CCFD_ERR_NOMEM;
		goto out;
	}
	long iv = 0, iid = 0;
	for (int e = 0; e < nblk && st == CCFD_OK; ++e) {
		long nin = 0;
		if (!fgets(line, sizeof(line), f) || sscanf(line, "%*d %*d %*d %ld", &nin) != 1 ||
		    nin < 0 || iid + nin > nv) {
			st = CCFD_ERR_MESH;
			break;
		}
		for (long i = 0; i < nin && st == CCFD_OK; ++i)
			if (!fgets(line, sizeof(line), f) || sscanf(line, "%ld", &ids[iid++]) != 1)
				st = CCFD_ERR_MESH;
		for (long i = 0; i < nin && st == CCFD_OK; ++i) {
			double x, y;
			if (!fgets(line, sizeof(line), f) || sscanf(line, "%lg %lg", &x, &y) != 2 ||
			    ids[iv] != iv + 1) {
				st = CCFD_ERR_MESH; /* "NodeID does not match Node Position" */
				break;
			}
			nodes[2 * iv] = x;
			nodes[2 * iv + 1] = y;
			iv++;
		}
	}
	free(ids);
	if (st != CCFD_OK)
		goto out;
	rewind(f);
	while (fgets(line, sizeof(line), f))
		if (!strcmp(line, "$Elements\n")) {
			if (!fgets(line, sizeof(line), f) || sscanf(line, "%d %ld", &nblk, &ne) != 2)
				ne = 0;
			break;
		}
	if (ne <= 0) {
		st = CCFD_ERR_MESH; /* "No Elements in Mesh file" */
		goto out;
	}
	tria = malloc(sizeof(long) * 4 * ne);
	quad = malloc(sizeof(long) * 5 * ne);
	bc = malloc(sizeof(long) * 3 * ne);
	if (!tria || !quad || !bc) {
		st = CCFD_ERR_NOMEM;
		goto out;
	}
	for (int e = 0; e < nblk && st == CCFD_OK; ++e) {
		int type = 0;
		long nin = 0;
		if (!fgets(line, sizeof(line), f) || sscanf(line, "%*d %*d %d %ld", &type, &nin) != 2 || nin < 0) {
			st = CCFD_ERR_MESH;
			break;
		}
		if (type < 1 || type > 3)
			continue;
		if ((type == 1 && e >= nptag) || nb + nt + nq + nin > ne) {
			st = CCFD_ERR_MESH;
			break;
		}
		for (long i = 0; i < nin; ++i) {
			long a[4];
			int want = type + 1, got;
			if (!fgets(line, sizeof(line), f)) {
				st = CCFD_ERR_MESH;
				break;
			}
			got = sscanf(line, "%*d %ld %ld %ld %ld", &a[0], &a[1], &a[2], &a[3]);
			if (got < want) {
				st = CCFD_ERR_MESH;
				break;
			}
			if (type == 1) {
				bc[3 * nb] = a[0] - 1;
				bc[3 * nb + 1] = a[1] - 1;
				bc[3 * nb + 2] = ptag[e];
				nb++;
			} else if (type == 2) {
				for (int k = 0; k < 3; ++k)
					tria[4 * nt + k] = a[k] - 1;
				tria[4 * nt + 3] = 1;
				nt++;
			} else {
				for (int k = 0; k < 4; ++k)
					quad[5 * nq + k] = a[k] - 1;
				quad[5 * nq + 4] = 1;
				nq++;
			}
		}
	}
	if (st == CCFD_OK && nt + nq == 0)
		st = CCFD_ERR_MESH;
out:
	free(ptag);
	if (st != CCFD_OK) {
		free(nodes); free(tria); free(quad); free(bc);
		return st;
	}
	*nodes_out = nodes;
	*n_nodes = nv;
	*tria_out = tria;
	*n_tria = nt;
	*quad_out = quad;
	*n_quad = nq;
	*bc_out = bc;
	*n_bc = nb;
	return CCFD_OK;
}

int ccfd_read_gmsh(const char *path, double **nodes_out, long *n_nodes,
		   long **tria_out, long *n_tria, long **quad_out, long *n_quad,
		   long **bc_out, long *n_bc)
{
	FILE *f = fopen(path, "r");
	if (!f)
		return CCFD_ERR_MESH;
	char line[1024];
	int fmt = 0;
	long nv = 0, ne = 0;
	double *nodes = NULL;
	long *tria = NULL, *quad = NULL, *bc = NULL;
	long nt = 0, nq = 0, nb = 0;
	int st = CCFD_OK;
	while (fgets(line, sizeof(line), f)) {
		if (!strcmp(line, "$MeshFormat\n")) {
			double v = 0;
			if (!fgets(line, sizeof(line), f) || sscanf(line, "%lg", &v) != 1) {
				st = CCFD_ERR_MESH;
				goto out;
			}
			fmt = (int)v;
			if (fmt == 4) {
				st = read_gmsh4(f, nodes_out, n_nodes, tria_out, n_tria, quad_out, n_quad,
						bc_out, n_bc);
				fclose(f);
				return st;
			}
			if (fmt != 2) {
				st = CCFD_ERR_MESH; /* "Wrong gmsh Mesh Format" */
				goto out;
			}
		} else if (!strcmp(line, "$Nodes\n")) {
			if (!fgets(line, sizeof(line), f) || sscanf(line, "%ld", &nv) != 1 || nv <= 0) {
				st = CCFD_ERR_MESH;
				goto out;
			}
			nodes = malloc(sizeof(double) * 2 * nv);
			if (!nodes) {
				st = CCFD_ERR_NOMEM;
				goto out;
			}
			for (long i = 0; i < nv; ++i) {
				long id;
				double x, y;
				if (!fgets(line, sizeof(line), f) ||
				    sscanf(line, "%ld %lg %lg", &id, &x, &y) != 3 || id != i + 1) {
					st = CCFD_ERR_MESH;
					goto out;
				}
				nodes[2 * i] = x;
				nodes[2 * i + 1] = y;
			}
		} else if (!strcmp(line, "$Elements\n")) {
			if (!fgets(line, sizeof(line), f) || sscanf(line, "%ld", &ne) != 1 || ne <= 0) {
				st = CCFD_ERR_MESH;
				goto out;
			}
			tria = malloc(sizeof(long) * 4 * ne);
			quad = malloc(sizeof(long) * 5 * ne);
			bc = malloc(sizeof(long) * 3 * ne);
			if (!tria || !quad || !bc) {
				st = CCFD_ERR_NOMEM;
				goto out;
			}
			for (long i = 0; i < ne; ++i) {
				if (!fgets(line, sizeof(line), f)) {
					st = CCFD_ERR_MESH;
					goto out;
				}
				long tok[16];
				int nt_ = 0;
				char *save = NULL;
				for (char *t = strtok_r(line, " \t\n", &save); t && nt_ < 16;
				     t = strtok_r(NULL, " \t\n", &save))
					tok[nt_++] = strtol(t, NULL, 10);
				if (nt_ < 4) {
					st = CCFD_ERR_MESH;
					goto out;
				}
				long type = tok[1], ntags = tok[2], pgroup = tok[3];
				long *nd = &tok[3 + ntags];
				int have = nt_ - 3 - (int)ntags;
				if (type == 1 && pgroup > 100 && have >= 2) {
					bc[3 * nb] = nd[0] - 1;
					bc[3 * nb + 1] = nd[1] - 1;
					bc[3 * nb + 2] = pgroup;
					nb++;
				} else if (type == 2 && have >= 3) {
					for (int k = 0; k < 3; ++k)
						tria[4 * nt + k] = nd[k] - 1;
					tria[4 * nt + 3] = pgroup;
					nt++;
				} else if (type == 3 && have >= 4) {
					for (int k = 0; k < 4; ++k)
						quad[5 * nq + k] = nd[k] - 1;
					quad[5 * nq + 4] = pgroup;
					nq++;
				}
			}
		}
	}
	if (!nodes || (nt + nq) == 0)
		st = CCFD_ERR_MESH;
out:
	fclose(f);
	if (st != CCFD_OK) {
		free(nodes); free(tria); free(quad); free(bc);
		return st;
	}
	*nodes_out = nodes;
	*n_nodes = nv;
	*tria_out = tria;
	*n_tria = nt;
	*quad_out = quad;
	*n_quad = nq;
	*bc_out = bc;
	*n_bc = nb;
	return CCFD_OK;
}

/* ------------------------------------------------------------ EMC2 */
/* next line of f that contains `key`, scanning from the start and stopping at
 * a line with "End" (the section search of readEMC2); the count on the line
 * after it, or -1 */
static long emc2_section(FILE *f, const char *key, char *line, size_t n)
{
	rewind(f);
	while (fgets(line, (int)n, f)) {
		if (strstr(line, key)) {
			long c = -1;
			if (!fgets(line, (int)n, f) || sscanf(line, "%ld", &c) != 1)
				return -1;
			return c;
		} else if (strstr(line, "End")) {
			break;
		}
	}
	return -1;
}

int ccfd_read_emc2(const char *path, double **nodes_out, long *n_nodes,
		   long **tria_out, long *n_tria, long **quad_out, long *n_quad,
		   long **bc_out, long *n_bc)
{
	/* readEMC2, src/mesh.c:1004-1139: Vertices (x y), Edges (a b ref;
	 * ref 0 is not a boundary edge and is dropped), Triangles (a b c ref),
	 * Quadrangles (a b c d ref); the element reference is its domain */
	FILE *f = fopen(path, "r");
	if (!f)
		return CCFD_ERR_MESH; /* "Could not find Mesh File" */
	char line[1024];
	int st = CCFD_OK;
	double *nodes = NULL;
	long *tria = NULL, *quad = NULL, *bc = NULL;
	long nv = emc2_section(f, "Vertices", line, sizeof(line)), ne = 0, nb = 0, nt = 0, nq = 0;
	if (nv <= 0) {
		st = CCFD_ERR_MESH;
		goto out;
	}
	nodes = malloc(sizeof(double) * 2 * nv);
	if (!nodes) {
		st = CCFD_ERR_NOMEM;
		goto out;
	}
	for (long i = 0; i < nv; ++i)
		if (!fgets(line, sizeof(line), f) || sscanf(line, "%lg %lg", &nodes[2 * i], &nodes[2 * i + 1]) != 2) {
			st = CCFD_ERR_MESH;
			goto out;
		}
	ne = emc2_section(f, "Edges", line, sizeof(line));
	if (ne < 0)
		ne = 0;
	bc = malloc(sizeof(long) * 3 * (ne > 0 ? ne : 1));
	if (!bc) {
		st = CCFD_ERR_NOMEM;
		goto out;
	}
	for (long i = 0; i < ne; ++i) {
		long a, b, r;
		if (!fgets(line, sizeof(line), f) || sscanf(line, "%ld %ld %ld", &a, &b, &r) != 3) {
			st = CCFD_ERR_MESH;
			goto out;
		}
		if (r != 0) {
			bc[3 * nb] = a - 1;
			bc[3 * nb + 1] = b - 1;
			bc[3 * nb + 2] = r;
			nb++;
		}
	}
	nt = emc2_section(f, "Triangles", line, sizeof(line));
	if (nt < 0)
		nt = 0;
	tria = malloc(sizeof(long) * 4 * (nt > 0 ? nt : 1));
	if (!tria) {
		st = CCFD_ERR_NOMEM;
		goto out;
	}
	for (long i = 0; i < nt; ++i) {
		long a[4];
		if (!fgets(line, sizeof(line), f) || sscanf(line, "%ld %ld %ld %ld", &a[0], &a[1], &a[2], &a[3]) != 4) {
			st = CCFD_ERR_MESH;
			goto out;
		}
		for (int k = 0; k < 3; ++k)
			tria[4 * i + k] = a[k] - 1;
		tria[4 * i + 3] = a[3];
	}
	nq = emc2_section(f, "Quadrangles", line, sizeof(line));
	if (nq < 0)
		nq = 0;
	quad = malloc(sizeof(long) * 5 * (nq > 0 ? nq : 1));
	if (!quad) {
		st = CCFD_ERR_NOMEM;
		goto out;
	}
	for (long i = 0; i < nq; ++i) {
		long a[5];
		if (!fgets(line, sizeof(line), f) ||
		    sscanf(line, "%ld %ld %ld %ld %ld", &a[0], &a[1], &a[2], &a[3], &a[4]) != 5) {
			st = CCFD_ERR_MESH;
			goto out;
		}
		for (int k = 0; k < 4; ++k)
			quad[5 * i + k] = a[k] - 1;
		quad[5 * i + 4] = a[4];
	}
	if (nt + nq == 0)
		st = CCFD_ERR_MESH;
out:
	fclose(f);
	if (st != CCFD_OK) {
		free(nodes); free(tria); free(quad); free(bc);
		return st;
	}
	*nodes_out = nodes;
	*n_nodes = nv;
	*tria_out = tria;
	*n_tria = nt;
	*quad_out = quad;
	*n_quad = nq;
	*bc_out = bc;
	*n_bc = nb;
	return CCFD_OK;
}
