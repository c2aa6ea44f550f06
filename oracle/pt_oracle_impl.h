/*
 * Oracle implementation, included by pt_oracle.c once per real type with
 * REAL (double or float) and SFX(name) (name suffix) defined.
 *
 * TEST INFRASTRUCTURE ONLY (see pt_oracle.h).
 *
 * The algorithm is the reference's (src/pt.c:40-1050; src/ptmp.c is the same
 * text in float): for every occupied triple the connected triples amplitude
 * W(abc) is assembled from contractions of doubles amplitudes with OVVV
 * integrals (contraction over a virtual index, src/pt.c:40-99) and with OOVO
 * integrals (contraction over an occupied index, src/pt.c:101-160), each
 * contraction being antisymmetrised into W with the index permutation and
 * sign the reference uses; the disconnected term V (src/pt.c:162-185) and the
 * denominator D give the triple's energy  sum W(W-V)/D  ((T)) or
 * sum (L-V)R/D  ((fT)).  The contractions are plain loop nests here (no BLAS),
 * and the permutation/sign data of each term is written as a table.
 */

/* Y[x][n] = sum_d A[x*lda + d] * B[d*ldb + n]   (x < m, n < nn, d < kd).
 * The OVVV-type contraction of src/pt.c:40-99: one amplitude slice (rows =
 * first virtual, columns = contracted virtual d) times one OVVV slice (rows d,
 * columns = the remaining virtual pair, packed b>c or full). */
static void SFX(contract_vir)(size_t m, size_t nn, size_t kd, const REAL *A,
    size_t lda, const REAL *B, size_t ldb, REAL *Y)
{
	for (size_t x = 0; x < m; x++) {
		REAL *y = Y + x*nn;
		for (size_t n = 0; n < nn; n++)
			y[n] = 0;
		for (size_t d = 0; d < kd; d++) {
			const REAL a = A[x*lda + d];
			const REAL *b = B + d*ldb;
			for (size_t n = 0; n < nn; n++)
				y[n] += a * b[n];
		}
	}
}

/* Zt[x][r] = sum_l B[x*ldb + l] * A[l*lda + r]   (x < nx, r < nr, l < kl).
 * The OOVO-type contraction of src/pt.c:101-160, stored transposed: the
 * reference's output element abc1[r + x*nr] is Zt[x][r] here. */
static void SFX(contract_occ)(size_t nx, size_t nr, size_t kl, const REAL *A,
    size_t lda, const REAL *B, size_t ldb, REAL *Zt)
{
	for (size_t x = 0; x < nx; x++) {
		REAL *z = Zt + x*nr;
		for (size_t r = 0; r < nr; r++)
			z[r] = 0;
		for (size_t l = 0; l < kl; l++) {
			const REAL b = B[x*ldb + l];
			const REAL *a = A + l*lda;
			for (size_t r = 0; r < nr; r++)
				z[r] += b * a[r];
		}
	}
}

static size_t SFX(pair)(size_t m, size_t n)   /* m > n, packed b>c index */
{
	return m*(m-1)/2 + n;
}

/* ---------------- same-spin triples (i<j<k, a>b>c) ----------------------- */

/* Blocks of one same-spin case: amplitudes tau[o][o][v][v], OVVV packed
 * [o][v][v(v-1)/2], OOVO [o][o][v][o]. */
struct SFX(aaa_in) {
	size_t o, v;
	const REAL *tau, *ovvv, *oovo;
};

/* W[(a*v+b)*v+c] for a>b>c: src/pt.c:236-290 (and 588-696 for (fT)). */
static void SFX(connected_aaa)(const struct SFX(aaa_in) *in, size_t i,
    size_t j, size_t k, REAL *W, REAL *Y)
{
	const size_t o = in->o, v = in->v, np = v*(v-1)/2;
	/* OVVV terms: (p,q,r) -> tau[p][q] x ovvv[r]; pattern +Y[c|ab]-Y[b|ac]+Y[a|bc]
	 * scaled by sign (src/pt.c:236-261). */
	const size_t vt[3][3] = { {i, j, k}, {i, k, j}, {k, j, i} };
	const int vs[3] = { +1, -1, -1 };
	/* OOVO terms: (p,q,r) -> tau[p][l] x oovo[q][r]; pattern
	 * +Z[bc|a]-Z[ac|b]-Z[ba|c] scaled by sign (src/pt.c:263-290). */
	const size_t ot[3][3] = { {i, j, k}, {j, i, k}, {k, j, i} };
	const int os[3] = { +1, -1, -1 };

	for (size_t x = 0; x < v*v*v; x++)
		W[x] = 0;
	for (int t = 0; t < 3; t++) {
		const size_t p = vt[t][0], q = vt[t][1], r = vt[t][2];
		SFX(contract_vir)(v, np, v, in->tau + (p*o+q)*v*v, v,
		    in->ovvv + r*v*np, np, Y);
		const REAL s = (REAL)vs[t];
		for (size_t a = 0; a < v; a++)
		for (size_t b = 0; b < a; b++)
		for (size_t c = 0; c < b; c++)
			W[(a*v+b)*v+c] += s * (Y[c*np + SFX(pair)(a, b)]
			    - Y[b*np + SFX(pair)(a, c)] + Y[a*np + SFX(pair)(b, c)]);
	}
	for (int t = 0; t < 3; t++) {
		const size_t p = ot[t][0], q = ot[t][1], r = ot[t][2];
		SFX(contract_occ)(v, v*v, o, in->tau + p*o*v*v, v*v,
		    in->oovo + (q*o+r)*v*o, o, Y);
		const REAL s = (REAL)os[t];
		for (size_t a = 0; a < v; a++)
		for (size_t b = 0; b < a; b++)
		for (size_t c = 0; c < b; c++)
			W[(a*v+b)*v+c] += s * (Y[a*v*v + b*v+c]
			    - Y[b*v*v + a*v+c] - Y[c*v*v + b*v+a]);
	}
}

/* Disconnected term of same-spin triples, src/pt.c:162-175:
 * sum over (p,q,r) in {(i,j,k)+,(j,i,k)-,(k,j,i)-} and
 * (x;y,z) in {(a;b,c)+,(b;a,c)-,(c;b,a)-} of ov[p,x] * oovv[q,r,y,z]. */
static REAL SFX(disc_aaa)(size_t o, size_t v, const REAL *ov, const REAL *oovv,
    size_t i, size_t j, size_t k, size_t a, size_t b, size_t c)
{
	const size_t P[3][3] = { {i, j, k}, {j, i, k}, {k, j, i} };
	const size_t X[3][3] = { {a, b, c}, {b, a, c}, {c, b, a} };
	const REAL S[3] = { 1, -1, -1 };
	REAL sum = 0;
	for (int u = 0; u < 3; u++)
	for (int w = 0; w < 3; w++)
		sum += S[u] * S[w] * ov[P[u][0]*v + X[w][0]] *
		    oovv[((P[u][1]*o + P[u][2])*v + X[w][1])*v + X[w][2]];
	return sum;
}

/* ---------------- mixed-spin triples (i<j alpha, k beta) ----------------- */

/* Blocks of one mixed-spin case (src/pt.c:304-313 argument list).
 * tau_aa[oa][oa][va][va] tau_ab[oa][ob][va][vb] tau_ba[ob][oa][vb][va]
 * ovvv_aa[oa][va][va(va-1)/2] ovvv_ab[oa][vb][va][vb] ovvv_ba[ob][va][vb][va]
 * oovo_aa[oa][oa][va][oa] oovo_ab[oa][ob][va][ob] oovo_ba[ob][oa][vb][oa] */
struct SFX(aab_in) {
	size_t oa, va, ob, vb;
	const REAL *tau_aa, *tau_ab, *tau_ba;
	const REAL *ovvv_aa, *ovvv_ab, *ovvv_ba;
	const REAL *oovo_aa, *oovo_ab, *oovo_ba;
};

/* W[(a*va+b)*vb+c] for a>b (alpha), c (beta): src/pt.c:361-432. */
static void SFX(connected_aab)(const struct SFX(aab_in) *in, size_t i,
    size_t j, size_t k, REAL *W, REAL *Y)
{
	const size_t oa = in->oa, va = in->va, ob = in->ob, vb = in->vb;
	const size_t np = va*(va-1)/2;
	size_t a, b, c;

	for (size_t x = 0; x < va*va*vb; x++)
		W[x] = 0;
#define LOOP for (a = 0; a < va; a++) for (b = 0; b < a; b++) for (c = 0; c < vb; c++)
#define WW W[(a*va+b)*vb+c]
	/* tau_aa[i][j] x ovvv_ba[k]: Y[x][m*va+n], m beta (src/pt.c:361-367) */
	SFX(contract_vir)(va, vb*va, va, in->tau_aa + (i*oa+j)*va*va, va,
	    in->ovvv_ba + k*va*vb*va, vb*va, Y);
	LOOP WW += -Y[a*vb*va + c*va+b] + Y[b*vb*va + c*va+a];
	/* tau_ab[i][k] x ovvv_ab[j] (src/pt.c:369-375) */
	SFX(contract_vir)(va, va*vb, vb, in->tau_ab + (i*ob+k)*va*vb, vb,
	    in->ovvv_ab + j*vb*va*vb, va*vb, Y);
	LOOP WW += -Y[a*va*vb + b*vb+c] + Y[b*va*vb + a*vb+c];
	/* tau_ab[j][k] x ovvv_ab[i] (src/pt.c:377-383) */
	SFX(contract_vir)(va, va*vb, vb, in->tau_ab + (j*ob+k)*va*vb, vb,
	    in->ovvv_ab + i*vb*va*vb, va*vb, Y);
	LOOP WW += Y[a*va*vb + b*vb+c] - Y[b*va*vb + a*vb+c];
	/* tau_ba[k][j] x ovvv_aa[i] and tau_ba[k][i] x ovvv_aa[j], packed pair
	 * (src/pt.c:385-392) */
	SFX(contract_vir)(vb, np, va, in->tau_ba + (k*oa+j)*vb*va, va,
	    in->ovvv_aa + i*va*np, np, Y);
	LOOP WW += -Y[c*np + SFX(pair)(a, b)];
	SFX(contract_vir)(vb, np, va, in->tau_ba + (k*oa+i)*vb*va, va,
	    in->ovvv_aa + j*va*np, np, Y);
	LOOP WW += Y[c*np + SFX(pair)(a, b)];
	/* oovo_ba[k][j] x tau_aa[i][l]: Zt[x beta][m*va+n] (src/pt.c:394-406) */
	SFX(contract_occ)(vb, va*va, oa, in->tau_aa + i*oa*va*va, va*va,
	    in->oovo_ba + (k*oa+j)*vb*oa, oa, Y);
	LOOP WW += -Y[c*va*va + a*va+b];
	SFX(contract_occ)(vb, va*va, oa, in->tau_aa + j*oa*va*va, va*va,
	    in->oovo_ba + (k*oa+i)*vb*oa, oa, Y);
	LOOP WW += Y[c*va*va + a*va+b];
	/* oovo_ab[j][k] x tau_ab[i][l] (src/pt.c:408-414) */
	SFX(contract_occ)(va, va*vb, ob, in->tau_ab + i*ob*va*vb, va*vb,
	    in->oovo_ab + (j*ob+k)*va*ob, ob, Y);
	LOOP WW += -Y[b*va*vb + a*vb+c] + Y[a*va*vb + b*vb+c];
	/* oovo_ab[i][k] x tau_ab[j][l] (src/pt.c:416-422) */
	SFX(contract_occ)(va, va*vb, ob, in->tau_ab + j*ob*va*vb, va*vb,
	    in->oovo_ab + (i*ob+k)*va*ob, ob, Y);
	LOOP WW += -Y[a*va*vb + b*vb+c] + Y[b*va*vb + a*vb+c];
	/* oovo_aa[j][i] x tau_ba[k][l]: Zt[x alpha][m*va+n], m beta
	 * (src/pt.c:424-432) */
	SFX(contract_occ)(va, vb*va, oa, in->tau_ba + k*oa*vb*va, vb*va,
	    in->oovo_aa + (j*oa+i)*va*oa, oa, Y);
	LOOP WW += -Y[b*vb*va + c*va+a] + Y[a*vb*va + c*va+b];
#undef LOOP
#undef WW
}

/* Disconnected term of mixed-spin triples, src/pt.c:177-185 and 433-442:
 * ov1/ov2 act on the alpha index pairs (i|a etc.) with the [oa][ob][va][vb]
 * oovv-like slice g_ab, the beta pair (k|c) with the [oa][oa][va][va] g_aa. */
static REAL SFX(disc_aab)(size_t oa, size_t va, size_t ob, size_t vb,
    const REAL *ov_a, const REAL *ov_b, const REAL *g_ab, const REAL *g_aa,
    size_t i, size_t j, size_t k, size_t a, size_t b, size_t c)
{
#define GAB(p, q, x, y) g_ab[(((p)*ob + (q))*va + (x))*vb + (y)]
	REAL sum = ov_a[i*va+a] * GAB(j, k, b, c);
	sum -= ov_a[i*va+b] * GAB(j, k, a, c);
	sum -= ov_a[j*va+a] * GAB(i, k, b, c);
	sum += ov_a[j*va+b] * GAB(i, k, a, c);
	sum += ov_b[k*vb+c] * g_aa[((j*oa + i)*va + b)*va + a];
#undef GAB
	return sum;
}

/* ---------------- energies ----------------------------------------------- */

/* One same-spin case.  pt: e = sum W(W-V)/D with V from (ov1,g1)+(ov2,g2);
 * ft: e = sum (L-V)R/D.  R == NULL selects (T). */
struct SFX(aaa_case) {
	struct SFX(aaa_in) L, R;   /* R.tau == NULL for (T) */
	const REAL *d_ov, *ov1, *g1, *ov2, *g2;
};

static double SFX(triple_aaa)(const struct SFX(aaa_case) *cs, size_t i,
    size_t j, size_t k, REAL *W, REAL *W2, REAL *Y)
{
	const size_t o = cs->L.o, v = cs->L.v;
	double e = 0;
	SFX(connected_aaa)(&cs->L, i, j, k, W, Y);
	if (cs->R.tau)
		SFX(connected_aaa)(&cs->R, i, j, k, W2, Y);
	for (size_t a = 0; a < v; a++)
	for (size_t b = 0; b < a; b++)
	for (size_t c = 0; c < b; c++) {
		const REAL dn = cs->d_ov[i*v+a] + cs->d_ov[j*v+b] + cs->d_ov[k*v+c];
		const REAL x = SFX(disc_aaa)(o, v, cs->ov1, cs->g1, i, j, k, a, b, c)
		    + SFX(disc_aaa)(o, v, cs->ov2, cs->g2, i, j, k, a, b, c);
		const REAL w = W[(a*v+b)*v+c];
		const REAL r = cs->R.tau ? W2[(a*v+b)*v+c] : w;
		e += (w - x) * r / dn;
	}
	return e;
}

struct SFX(aab_case) {
	struct SFX(aab_in) L, R;   /* R.tau_aa == NULL for (T) */
	const REAL *d_a, *d_b;
	const REAL *ov1_a, *ov1_b, *g1_ab, *g1_aa;
	const REAL *ov2_a, *ov2_b, *g2_ab, *g2_aa;
};

static double SFX(triple_aab)(const struct SFX(aab_case) *cs, size_t i,
    size_t j, size_t k, REAL *W, REAL *W2, REAL *Y)
{
	const size_t oa = cs->L.oa, va = cs->L.va, ob = cs->L.ob, vb = cs->L.vb;
	double e = 0;
	SFX(connected_aab)(&cs->L, i, j, k, W, Y);
	if (cs->R.tau_aa)
		SFX(connected_aab)(&cs->R, i, j, k, W2, Y);
	for (size_t a = 0; a < va; a++)
	for (size_t b = 0; b < a; b++)
	for (size_t c = 0; c < vb; c++) {
		const REAL dn = cs->d_a[i*va+a] + cs->d_a[j*va+b] + cs->d_b[k*vb+c];
		const REAL x = SFX(disc_aab)(oa, va, ob, vb, cs->ov1_a, cs->ov1_b,
		    cs->g1_ab, cs->g1_aa, i, j, k, a, b, c)
		    + SFX(disc_aab)(oa, va, ob, vb, cs->ov2_a, cs->ov2_b,
		    cs->g2_ab, cs->g2_aa, i, j, k, a, b, c);
		const REAL w = W[(a*va+b)*vb+c];
		const REAL r = cs->R.tau_aa ? W2[(a*va+b)*vb+c] : w;
		e += (w - x) * r / dn;
	}
	return e;
}

/* Triple lists in the reference's order (src/pt.c:210-221, 333-344). */
static size_t SFX(list_aaa)(size_t o, size_t *ijk)
{
	size_t n = 0;
	for (size_t i = 0; i < o; i++)
	for (size_t j = i+1; j < o; j++)
	for (size_t k = j+1; k < o; k++, n++)
		if (ijk) { ijk[3*n] = i; ijk[3*n+1] = j; ijk[3*n+2] = k; }
	return n;
}

static size_t SFX(list_aab)(size_t oa, size_t ob, size_t *ijk)
{
	size_t n = 0;
	for (size_t i = 0; i < oa; i++)
	for (size_t j = i+1; j < oa; j++)
	for (size_t k = 0; k < ob; k++, n++)
		if (ijk) { ijk[3*n] = i; ijk[3*n+1] = j; ijk[3*n+2] = k; }
	return n;
}

static void *SFX(xalloc)(size_t n)
{
	void *p = malloc(n ? n : 1);
	if (p == NULL) {
		fprintf(stderr, "oracle: out of memory (%zu bytes)\n", n);
		abort();
	}
	return p;
}

/* Per-triple energies of the same-spin case into part[] (triple order). */
static size_t SFX(run_aaa)(const struct SFX(aaa_case) *cs, double *part,
    size_t cap)
{
	const size_t o = cs->L.o, v = cs->L.v;
	if (o == 0 || v == 0)
		return 0;
	const size_t nt = SFX(list_aaa)(o, NULL);
	size_t *ijk = SFX(xalloc)(3*nt*sizeof(size_t) + 1);
	SFX(list_aaa)(o, ijk);
	#pragma omp parallel
	{
		REAL *W = SFX(xalloc)(3*v*v*v*sizeof(REAL));
		REAL *W2 = W + v*v*v, *Y = W2 + v*v*v;
		#pragma omp for schedule(dynamic)
		for (size_t t = 0; t < nt; t++) {
			double e = SFX(triple_aaa)(cs, ijk[3*t], ijk[3*t+1],
			    ijk[3*t+2], W, W2, Y);
			if (t < cap)
				part[t] = e;
		}
		free(W);
	}
	free(ijk);
	return nt;
}

static size_t SFX(run_aab)(const struct SFX(aab_case) *cs, double *part,
    size_t cap)
{
	const size_t oa = cs->L.oa, va = cs->L.va, ob = cs->L.ob, vb = cs->L.vb;
	if (oa == 0 || va == 0 || ob == 0 || vb == 0)
		return 0;
	const size_t nt = SFX(list_aab)(oa, ob, NULL);
	const size_t vm = va > vb ? va : vb;
	size_t *ijk = SFX(xalloc)(3*nt*sizeof(size_t) + 1);
	SFX(list_aab)(oa, ob, ijk);
	#pragma omp parallel
	{
		REAL *W = SFX(xalloc)(3*vm*vm*vm*sizeof(REAL));
		REAL *W2 = W + vm*vm*vm, *Y = W2 + vm*vm*vm;
		#pragma omp for schedule(dynamic)
		for (size_t t = 0; t < nt; t++) {
			double e = SFX(triple_aab)(cs, ijk[3*t], ijk[3*t+1],
			    ijk[3*t+2], W, W2, Y);
			if (t < cap)
				part[t] = e;
		}
		free(W);
	}
	free(ijk);
	return nt;
}

/* Fixed-order sum of a case's per-triple energies. */
static double SFX(sum_aaa)(const struct SFX(aaa_case) *cs)
{
	const size_t o = cs->L.o;
	const size_t nt = (o && cs->L.v) ? SFX(list_aaa)(o, NULL) : 0;
	double *part = SFX(xalloc)((nt+1)*sizeof(double)), e = 0;
	SFX(run_aaa)(cs, part, nt);
	for (size_t t = 0; t < nt; t++)
		e += part[t];
	free(part);
	return e;
}

static double SFX(sum_aab)(const struct SFX(aab_case) *cs)
{
	const size_t oa = cs->L.oa, ob = cs->L.ob;
	const size_t nt = (oa && ob && cs->L.va && cs->L.vb) ?
	    SFX(list_aab)(oa, ob, NULL) : 0;
	double *part = SFX(xalloc)((nt+1)*sizeof(double)), e = 0;
	SFX(run_aab)(cs, part, nt);
	for (size_t t = 0; t < nt; t++)
		e += part[t];
	free(part);
	return e;
}

/* ---------------- spin-block drivers ------------------------------------- */

/* Offsets of the four spin blocks of a packed argument (src/pt.c:487-512). */
struct SFX(blocks) {
	const REAL *aaaa, *abab, *bbbb, *baba;
};

static struct SFX(blocks) SFX(split4)(const REAL *p, size_t s_aaaa,
    size_t s_abab, size_t s_bbbb)
{
	struct SFX(blocks) b;
	b.aaaa = p;
	b.abab = p + s_aaaa;
	b.bbbb = b.abab + s_abab;
	b.baba = b.bbbb + s_bbbb;
	return b;
}

/* Sizes of the four spin blocks of each tensor kind. */
#define OOVV_SZ(o1, o2, v1, v2) ((o1)*(o2)*(v1)*(v2))
#define OOVO_SZ(o1, o2, v1)     ((o1)*(o2)*(v1)*(o2))
#define OVVV_AA_SZ(o, v)        ((o)*(v)*(v)*((v)-1)/2)

static struct SFX(aab_in) SFX(mk_aab)(size_t oa, size_t va, size_t ob,
    size_t vb, const REAL *taa, const REAL *tab, const REAL *tba,
    const REAL *vaa, const REAL *vab, const REAL *vba, const REAL *oaa,
    const REAL *oab, const REAL *oba)
{
	struct SFX(aab_in) in;
	in.oa = oa; in.va = va; in.ob = ob; in.vb = vb;
	in.tau_aa = taa; in.tau_ab = tab; in.tau_ba = tba;
	in.ovvv_aa = vaa; in.ovvv_ab = vab; in.ovvv_ba = vba;
	in.oovo_aa = oaa; in.oovo_ab = oab; in.oovo_ba = oba;
	return in;
}

/* (T), any spin: the four cases of src/pt.c:514-529 (restricted calls only
 * the first and third with beta == alpha, src/pt.c:469-473). */
static double SFX(pt_cases)(int unrestricted, size_t oa, size_t va, size_t ob,
    size_t vb, const REAL *d_ov, const REAL *f_ov, const REAL *t1,
    const REAL *t2, const REAL *i_oovo, const REAL *i_oovv,
    const REAL *i_ovvv)
{
	const REAL *d_b = unrestricted ? d_ov + oa*va : d_ov;
	const REAL *f_b = unrestricted ? f_ov + oa*va : f_ov;
	const REAL *t1_b = unrestricted ? t1 + oa*va : t1;
	struct SFX(blocks) T = SFX(split4)(t2, OOVV_SZ(oa, oa, va, va),
	    OOVV_SZ(oa, ob, va, vb), OOVV_SZ(ob, ob, vb, vb));
	struct SFX(blocks) G = SFX(split4)(i_oovv, OOVV_SZ(oa, oa, va, va),
	    OOVV_SZ(oa, ob, va, vb), OOVV_SZ(ob, ob, vb, vb));
	struct SFX(blocks) O = SFX(split4)(i_oovo, OOVO_SZ(oa, oa, va),
	    OOVO_SZ(oa, ob, va), OOVO_SZ(ob, ob, vb));
	struct SFX(blocks) V = SFX(split4)(i_ovvv, OVVV_AA_SZ(oa, va),
	    oa*vb*va*vb, OVVV_AA_SZ(ob, vb));
	if (!unrestricted) {   /* restricted: baba aliases abab (src/pt.c:471-473) */
		T.baba = T.abab; G.baba = G.abab; O.baba = O.abab; V.baba = V.abab;
	}
	double e = 0;
	struct SFX(aaa_case) ca;
	memset(&ca, 0, sizeof(ca));
	ca.L.o = oa; ca.L.v = va; ca.L.tau = T.aaaa; ca.L.ovvv = V.aaaa;
	ca.L.oovo = O.aaaa;
	ca.d_ov = d_ov; ca.ov1 = t1; ca.g1 = G.aaaa; ca.ov2 = f_ov; ca.g2 = T.aaaa;
	e += SFX(sum_aaa)(&ca);
	if (unrestricted) {
		ca.L.o = ob; ca.L.v = vb; ca.L.tau = T.bbbb; ca.L.ovvv = V.bbbb;
		ca.L.oovo = O.bbbb;
		ca.d_ov = d_b; ca.ov1 = t1_b; ca.g1 = G.bbbb; ca.ov2 = f_b;
		ca.g2 = T.bbbb;
		e += SFX(sum_aaa)(&ca);
	}
	struct SFX(aab_case) cb;
	memset(&cb, 0, sizeof(cb));
	cb.L = SFX(mk_aab)(oa, va, ob, vb, T.aaaa, T.abab, T.baba, V.aaaa,
	    V.abab, V.baba, O.aaaa, O.abab, O.baba);
	cb.d_a = d_ov; cb.d_b = d_b;
	cb.ov1_a = t1; cb.ov1_b = t1_b; cb.g1_ab = G.abab; cb.g1_aa = G.aaaa;
	cb.ov2_a = f_ov; cb.ov2_b = f_b; cb.g2_ab = T.abab; cb.g2_aa = T.aaaa;
	e += SFX(sum_aab)(&cb);
	if (unrestricted) {
		cb.L = SFX(mk_aab)(ob, vb, oa, va, T.bbbb, T.baba, T.abab, V.bbbb,
		    V.baba, V.abab, O.bbbb, O.baba, O.abab);
		cb.d_a = d_b; cb.d_b = d_ov;
		cb.ov1_a = t1_b; cb.ov1_b = t1; cb.g1_ab = G.baba; cb.g1_aa = G.bbbb;
		cb.ov2_a = f_b; cb.ov2_b = f_ov; cb.g2_ab = T.baba;
		cb.g2_aa = T.bbbb;
		e += SFX(sum_aab)(&cb);
	}
	return unrestricted ? e : 2.0 * e;
}

/* (fT), any spin: src/pt.c:958-966 (restricted) and 1023-1044. */
static double SFX(ft_cases)(int unrestricted, size_t oa, size_t va, size_t ob,
    size_t vb, const REAL *d_ov, const REAL *f2_ov, const REAL *l1,
    const REAL *t2, const REAL *l2, const REAL *i_oovv,
    const REAL *i2_t2f2_oovo, const REAL *i3_ovvv, const REAL *i6_oovo,
    const REAL *i7_ovvv)
{
	const REAL *d_b = unrestricted ? d_ov + oa*va : d_ov;
	const REAL *f_b = unrestricted ? f2_ov + oa*va : f2_ov;
	const REAL *l1_b = unrestricted ? l1 + oa*va : l1;
	const size_t s4v[3] = { OOVV_SZ(oa, oa, va, va), OOVV_SZ(oa, ob, va, vb),
	    OOVV_SZ(ob, ob, vb, vb) };
	const size_t s4o[3] = { OOVO_SZ(oa, oa, va), OOVO_SZ(oa, ob, va),
	    OOVO_SZ(ob, ob, vb) };
	const size_t s4w[3] = { OVVV_AA_SZ(oa, va), oa*vb*va*vb,
	    OVVV_AA_SZ(ob, vb) };
	struct SFX(blocks) T = SFX(split4)(t2, s4v[0], s4v[1], s4v[2]);
	struct SFX(blocks) L = SFX(split4)(l2, s4v[0], s4v[1], s4v[2]);
	struct SFX(blocks) G = SFX(split4)(i_oovv, s4v[0], s4v[1], s4v[2]);
	struct SFX(blocks) O2 = SFX(split4)(i2_t2f2_oovo, s4o[0], s4o[1], s4o[2]);
	struct SFX(blocks) O6 = SFX(split4)(i6_oovo, s4o[0], s4o[1], s4o[2]);
	struct SFX(blocks) V3 = SFX(split4)(i3_ovvv, s4w[0], s4w[1], s4w[2]);
	struct SFX(blocks) V7 = SFX(split4)(i7_ovvv, s4w[0], s4w[1], s4w[2]);
	if (!unrestricted) {
		T.baba = T.abab; L.baba = L.abab; G.baba = G.abab;
		O2.baba = O2.abab; O6.baba = O6.abab; V3.baba = V3.abab;
		V7.baba = V7.abab;
	}
	double e = 0;
	for (int spin = 0; spin < (unrestricted ? 2 : 1); spin++) {
		struct SFX(aaa_case) ca;
		memset(&ca, 0, sizeof(ca));
		const int b = spin == 1;
		ca.L.o = ca.R.o = b ? ob : oa;
		ca.L.v = ca.R.v = b ? vb : va;
		ca.L.tau = b ? L.bbbb : L.aaaa;
		ca.L.ovvv = b ? V7.bbbb : V7.aaaa;
		ca.L.oovo = b ? O6.bbbb : O6.aaaa;
		ca.R.tau = b ? T.bbbb : T.aaaa;
		ca.R.ovvv = b ? V3.bbbb : V3.aaaa;
		ca.R.oovo = b ? O2.bbbb : O2.aaaa;
		ca.d_ov = b ? d_b : d_ov;
		ca.ov1 = b ? l1_b : l1;
		ca.g1 = b ? G.bbbb : G.aaaa;
		ca.ov2 = b ? f_b : f2_ov;
		ca.g2 = b ? L.bbbb : L.aaaa;
		e += SFX(sum_aaa)(&ca);
	}
	for (int spin = 0; spin < (unrestricted ? 2 : 1); spin++) {
		struct SFX(aab_case) cb;
		memset(&cb, 0, sizeof(cb));
		if (spin == 0) {
			cb.L = SFX(mk_aab)(oa, va, ob, vb, L.aaaa, L.abab, L.baba,
			    V7.aaaa, V7.abab, V7.baba, O6.aaaa, O6.abab, O6.baba);
			cb.R = SFX(mk_aab)(oa, va, ob, vb, T.aaaa, T.abab, T.baba,
			    V3.aaaa, V3.abab, V3.baba, O2.aaaa, O2.abab, O2.baba);
			cb.d_a = d_ov; cb.d_b = d_b;
			cb.ov1_a = l1; cb.ov1_b = l1_b; cb.g1_ab = G.abab;
			cb.g1_aa = G.aaaa;
			cb.ov2_a = f2_ov; cb.ov2_b = f_b; cb.g2_ab = L.abab;
			cb.g2_aa = L.aaaa;
		} else {
			cb.L = SFX(mk_aab)(ob, vb, oa, va, L.bbbb, L.baba, L.abab,
			    V7.bbbb, V7.baba, V7.abab, O6.bbbb, O6.baba, O6.abab);
			cb.R = SFX(mk_aab)(ob, vb, oa, va, T.bbbb, T.baba, T.abab,
			    V3.bbbb, V3.baba, V3.abab, O2.bbbb, O2.baba, O2.abab);
			cb.d_a = d_b; cb.d_b = d_ov;
			cb.ov1_a = l1_b; cb.ov1_b = l1; cb.g1_ab = G.baba;
			cb.g1_aa = G.bbbb;
			cb.ov2_a = f_b; cb.ov2_b = f2_ov; cb.g2_ab = L.baba;
			cb.g2_aa = L.bbbb;
		}
		e += SFX(sum_aab)(&cb);
	}
	return unrestricted ? e : 2.0 * e;
}
