/*
 * Oracle: CPU restatement of libpt's perturbative-triples energies.
 * TEST INFRASTRUCTURE ONLY -- see pt_oracle.h.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pt_oracle.h"

#define REAL double
#define SFX(name) name##_d
#include "pt_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL float
#define SFX(name) name##_f
#include "pt_oracle_impl.h"
#undef REAL
#undef SFX

double oracle_rpt(size_t oa, size_t va, const double *d_ov, const double *f_ov,
    const double *t1, const double *t2, const double *i_oovo,
    const double *i_oovv, const double *i_ovvv)
{
	return pt_cases_d(0, oa, va, oa, va, d_ov, f_ov, t1, t2, i_oovo, i_oovv,
	    i_ovvv);
}

double oracle_upt(size_t oa, size_t va, size_t ob, size_t vb,
    const double *d_ov, const double *f_ov, const double *t1, const double *t2,
    const double *i_oovo, const double *i_oovv, const double *i_ovvv)
{
	return pt_cases_d(1, oa, va, ob, vb, d_ov, f_ov, t1, t2, i_oovo, i_oovv,
	    i_ovvv);
}

double oracle_rft(size_t oa, size_t va, const double *d_ov,
    const double *f2_ov, const double *l1, const double *t2, const double *l2,
    const double *i_oovv, const double *i2_t2f2_oovo, const double *i3_ovvv,
    const double *i6_oovo, const double *i7_ovvv)
{
	return ft_cases_d(0, oa, va, oa, va, d_ov, f2_ov, l1, t2, l2, i_oovv,
	    i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv);
}

double oracle_uft(size_t oa, size_t va, size_t ob, size_t vb,
    const double *d_ov, const double *f2_ov, const double *l1,
    const double *t2, const double *l2, const double *i_oovv,
    const double *i2_t2f2_oovo, const double *i3_ovvv, const double *i6_oovo,
    const double *i7_ovvv)
{
	return ft_cases_d(1, oa, va, ob, vb, d_ov, f2_ov, l1, t2, l2, i_oovv,
	    i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv);
}

double oracle_rpt_mp(size_t oa, size_t va, const float *d_ov,
    const float *f_ov, const float *t1, const float *t2, const float *i_oovo,
    const float *i_oovv, const float *i_ovvv)
{
	return pt_cases_f(0, oa, va, oa, va, d_ov, f_ov, t1, t2, i_oovo, i_oovv,
	    i_ovvv);
}

double oracle_upt_mp(size_t oa, size_t va, size_t ob, size_t vb,
    const float *d_ov, const float *f_ov, const float *t1, const float *t2,
    const float *i_oovo, const float *i_oovv, const float *i_ovvv)
{
	return pt_cases_f(1, oa, va, ob, vb, d_ov, f_ov, t1, t2, i_oovo, i_oovv,
	    i_ovvv);
}

double oracle_rft_mp(size_t oa, size_t va, const float *d_ov,
    const float *f2_ov, const float *l1, const float *t2, const float *l2,
    const float *i_oovv, const float *i2_t2f2_oovo, const float *i3_ovvv,
    const float *i6_oovo, const float *i7_ovvv)
{
	return ft_cases_f(0, oa, va, oa, va, d_ov, f2_ov, l1, t2, l2, i_oovv,
	    i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv);
}

double oracle_uft_mp(size_t oa, size_t va, size_t ob, size_t vb,
    const float *d_ov, const float *f2_ov, const float *l1, const float *t2,
    const float *l2, const float *i_oovv, const float *i2_t2f2_oovo,
    const float *i3_ovvv, const float *i6_oovo, const float *i7_ovvv)
{
	return ft_cases_f(1, oa, va, ob, vb, d_ov, f2_ov, l1, t2, l2, i_oovv,
	    i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv);
}

size_t oracle_rpt_partials(int kind, size_t oa, size_t va, const double *d_ov,
    const double *f_ov, const double *t1, const double *t2,
    const double *i_oovo, const double *i_oovv, const double *i_ovvv,
    double *out, size_t cap)
{
	const double *t2_ab = t2 + oa*oa*va*va;
	const double *oovv_ab = i_oovv + oa*oa*va*va;
	const double *oovo_ab = i_oovo + oa*oa*oa*va;
	const double *ovvv_ab = i_ovvv + oa*va*va*(va-1)/2;
	if (kind == 0) {
		struct aaa_case_d ca;
		memset(&ca, 0, sizeof(ca));
		ca.L.o = oa; ca.L.v = va; ca.L.tau = t2; ca.L.ovvv = i_ovvv;
		ca.L.oovo = i_oovo;
		ca.d_ov = d_ov; ca.ov1 = t1; ca.g1 = i_oovv; ca.ov2 = f_ov; ca.g2 = t2;
		return run_aaa_d(&ca, out, cap);
	}
	struct aab_case_d cb;
	memset(&cb, 0, sizeof(cb));
	cb.L = mk_aab_d(oa, va, oa, va, t2, t2_ab, t2_ab, i_ovvv, ovvv_ab,
	    ovvv_ab, i_oovo, oovo_ab, oovo_ab);
	cb.d_a = d_ov; cb.d_b = d_ov;
	cb.ov1_a = t1; cb.ov1_b = t1; cb.g1_ab = oovv_ab; cb.g1_aa = i_oovv;
	cb.ov2_a = f_ov; cb.ov2_b = f_ov; cb.g2_ab = t2_ab; cb.g2_aa = t2;
	return run_aab_d(&cb, out, cap);
}
