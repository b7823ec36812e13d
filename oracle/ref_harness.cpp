/*
 * C-ABI harness over the UNMODIFIED reference sources (test infrastructure).
 *
 * oracle/build_ref.py compiles every file of the reference's library/ and
 * checks/ directories, exactly as they lie in the reference tree, together
 * with this file into oracle/_ref/libyahmc_ref_<config>.so, once per
 * compile-time physics configuration (-DNC, -DREPR_*, -DCLOVER_TERM,
 * -DUPDATE_EO, -DBC_*: programs/Makefile:6-45).  This file only sets the
 * reference's globals up the way programs/hmc.cpp:66-126 does and forwards
 * plain pointers to the reference's own functions, so the parity tests, the
 * golden-vector generator and the CPU baseline of bench.py can drive the
 * reference through ctypes.
 *
 * Nothing in the product links or loads this library.
 *
 * Host data layouts are the reference's own:
 *   spinor field : outer.vol4 x Spinor{ re[REPR_DIM][4], im[REPR_DIM][4] }  (include/spinor.h:7-9)
 *   fund links   : 4*outer.vol4 x suNg{ re[NC*NC], im[NC*NC] }  index 4*id+mu  (include/gaugefield.h:6-7)
 *   repr links   : 4*outer.vol4 x suNf                                         (include/gaugefield.h:9-10)
 *   momenta      : 4*outer.vol4 x suNa{ av[NG] }                                (include/gaugefield.h:12-13)
 *   clover term  : 4*outer.vol4 x suNf, clover force 6*outer.vol4 x suNf         (include/clover.h:12-16)
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif
/* reference headers last: include/gaugefield.h:6 defines a macro named link */
#include <global.h>
#include <settings.h>
#include <linalg.h>
#include <dirac.h>
#include <inverter.h>
#include <forces.h>
#include <clover.h>
#include <bcs.h>
#include <repr.h>
#include <random.h>
#include <spectrum.h>
#include <wilsonflow.h>
#include <logger.h>
#include <rational.h>
#include <staples.h>
#include <wilsonloop.h>
#include <checks.h>
#include <timing.h>
#include <update.h>
#include <mre.h>
#include <hirep.h>

/* defined in library/update.cpp without a header declaration */
double hamiltonian();
void reunitarize();
void reset_variables();
#include <integrator.h>
#include <approx.h>
/* defined in library/rational.cpp without a header declaration */
double residue(rational_app &data, int n);
void rescale(rational_app &data, double max);

static int harness_ready = 0;

static void wrap(SpinorField &sf, double *p)
{
	sf.ptr = (Spinor*)p;
	sf.allocated = false;
	spinor_type_default(sf);
}

/* view: 0 = the reference's default view, 1 = even, 2 = odd, 3 = full */
static void set_view(SpinorField &sf, int view)
{
	switch(view)
	{
		case 1: spinor_type_even(sf); break;
		case 2: spinor_type_odd(sf); break;
		case 3: spinor_type_full(sf); break;
		default: spinor_type_default(sf); break;
	}
}

static mvm_operator op_from_id(int op)
{
	switch(op)
	{
		case 0: return Dphi;
		case 1: return Hphi;
		case 2: return Hphi_sq;
		default: return 0;
	}
}

extern "C" {

/* Compile-time configuration of this build. */
void yref_info(int *out)
{
	out[0] = NC;
	out[1] = REPR_DIM;
	out[2] = NG;
	out[3] = REPR_ID;
#ifdef CLOVER_TERM
	out[4] = 1;
#else
	out[4] = 0;
#endif
#ifdef UPDATE_EO
	out[5] = 1;
#else
	out[5] = 0;
#endif
#if defined(BC_ANTIPERIODIC)
	out[6] = 1;
#elif defined(BC_OPEN)
	out[6] = 2;
#elif defined(BC_SF)
	out[6] = 3;
#else
	out[6] = 0;
#endif
	out[7] = (int)sizeof(Spinor);
	out[8] = (int)sizeof(suNf);
	out[9] = (int)sizeof(ldl_t);
}

/*
 * Set up geometry, representation, boundary conditions and the clover term
 * the way programs/hmc.cpp:72-117 does (single rank, border 1).  The lattice
 * sizes reach the reference through its own settings reader, so they are
 * written to a temporary cfg file first.  May be called once per process.
 */
int yref_init(int T, int X, int Y, int Z, double csw, double cf, int threads, int seed, int log_level)
{
	if(harness_ready)
	{
		return (global.dim_t == T && global.dim_x == X && global.dim_y == Y && global.dim_z == Z) ? 0 : -1;
	}

	char path[] = "/tmp/yahmc_oracle_cfgXXXXXX";
	int fd = mkstemp(path);
	if(fd < 0) return -2;
	FILE *fp = fdopen(fd, "w");
	fprintf(fp, "[lattice]\ndim_t = %d\ndim_x = %d\ndim_y = %d\ndim_z = %d\n", T, X, Y, Z);
	fprintf(fp, "[parallel]\nthreads = %d\nnp_t = 1\nnp_x = 1\nnp_y = 1\nnp_z = 1\n", threads);
	fprintf(fp, "[log]\nlevel = %d\n", log_level);
	fclose(fp);

	char *argv0 = (char*)"oracle";
	mp_init(1, &argv0);
	var_init(path);
	remove(path);
	if(log_level >= 0)
	{
		logger_init("", log_level);
	}
	geometry_init(1);
	mp_setup();
	rand_init(seed);
	repr_init();
	bcs_init(cf);
	clover_init(csw);
	gauge_field_init();
	gauge_field_set_unit();
	harness_ready = 1;
	return 0;
}

long yref_volume(void)
{
	return (long)outer.vol4;
}

void yref_set_threads(int threads)
{
#ifdef _OPENMP
	omp_set_num_threads(threads);
#endif
}

/* site[id].coord (t,x,y,z) and fw/bk neighbour tables, 4 ints each per site */
void yref_geometry(int *coord, int *fw, int *bk)
{
	for(int id = 0; id < outer.vol4; id++)
	{
		for(int mu = 0; mu < 4; mu++)
		{
			coord[4*id+mu] = site[id].coord[mu];
			fw[4*id+mu] = site[id].fw[mu];
			bk[4*id+mu] = site[id].bk[mu];
		}
	}
}

/* Fundamental links in, then the reference's represent_gauge_field() (repr.cpp:265-280). */
void yref_set_links(const double *fund)
{
	memcpy(gfield_fund, fund, sizeof(suNg)*4*outer.vol4);
	represent_gauge_field();
}

void yref_get_links(double *fund)
{
	memcpy(fund, gfield_fund, sizeof(suNg)*4*outer.vol4);
}

/* The reference's own random start (suNg::random, suNg.cpp:375-380) + gauge BCs + represent. */
void yref_set_random_links(void)
{
	gauge_field_set_random();
}

void yref_apply_bcs_on_gauge_field(void)
{
	apply_bcs_on_gauge_field();
}

void yref_get_repr_links(double *out)
{
	memcpy(out, gfield_repr, sizeof(suNf)*4*outer.vol4);
}

void yref_get_clover_term(double *out)
{
#ifdef CLOVER_TERM
	memcpy(out, cl_term, sizeof(suNf)*4*outer.vol4);
#endif
}

/* LDL factors for sigma = 4+mass (clover.cpp:307-328), both blocks, odd sites filled. */
void yref_get_ldl(double mass, double *out)
{
#ifdef CLOVER_TERM
	compute_ldl_decomp(4.0+mass);
	memcpy(out, cl_ldl, sizeof(ldl_t)*outer.vol4);
#endif
}

void yref_get_clover_force(double *out)
{
#ifdef CLOVER_TERM
	memcpy(out, cl_force, sizeof(suNf)*6*outer.vol4);
#endif
}

void yref_set_clover_force(const double *in)
{
#ifdef CLOVER_TERM
	memcpy(cl_force, in, sizeof(suNf)*6*outer.vol4);
#endif
}

void yref_get_generators(double *fund, double *repr)
{
	memcpy(fund, iTfund, sizeof(suNg)*NG);
	memcpy(repr, iTrepr, sizeof(suNf)*NG);
}

void yref_represent(double *repr_out, const double *fund_in, int count)
{
	represent_links((suNf*)repr_out, (suNg*)fund_in, count);
}

/* ---- Dirac operator (dirac.h) ---- */
void yref_Dphi_oe(double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); Dphi_oe(d, s); }
void yref_Dphi_eo(double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); Dphi_eo(d, s); }
void yref_Dphi_ee(double m, double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); Dphi_ee(m, d, s); }
void yref_Dphi_oo(double m, double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); Dphi_oo(m, d, s); }
void yref_Dphi_oo_inv(double m, double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); Dphi_oo_inv(m, d, s); }
void yref_Dphi(double m, double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); Dphi(m, d, s); }
void yref_Hphi(double m, double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); Hphi(m, d, s); }
void yref_Hphi_sq(double m, double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); Hphi_sq(m, d, s); }
int yref_mvm_get(void) { return mvm_get(); }
void yref_mvm_reset(void) { mvm_reset(); }

/* ---- clover (clover.h) ---- */
double yref_clover_logdet(double m) { return clover_logdet(m); }

/* ---- spinor linear algebra (linalg.h), view as in set_view() ---- */
void yref_spinor_random(double *a, int view) { SpinorField f; wrap(f, a); set_view(f, view); spinor_random(f); }
void yref_spinor_zero(double *a) { SpinorField f; wrap(f, a); spinor_zero(f); }
void yref_spinor_copy(double *a, double *b) { SpinorField f, g; wrap(f, a); wrap(g, b); spinor_copy(f, g); }
void yref_spinor_g5(double *a, int view) { SpinorField f; wrap(f, a); set_view(f, view); spinor_g5(f); }
double yref_spinor_sqnorm(double *a, int view) { SpinorField f; wrap(f, a); set_view(f, view); return spinor_sqnorm(f); }
double yref_spinor_product_re(double *a, double *b, int view)
{
	SpinorField f, g; wrap(f, a); wrap(g, b); set_view(f, view); set_view(g, view);
	return spinor_product_re(f, g);
}
void yref_spinor_product(double *a, double *b, int view, double *out)
{
	SpinorField f, g; wrap(f, a); wrap(g, b); set_view(f, view); set_view(g, view);
	complex c = spinor_product(f, g);
	out[0] = c.re; out[1] = c.im;
}
/* op: 0 add, 1 sub, 2 mulr, 3 mulc, 4 mulr_assign, 5 mulc_assign,
 *     6 mulr_add, 7 mulc_add, 8 mulr_sub, 9 mulc_sub */
void yref_spinor_axpy(int op, double *a, double re, double im, double *b, int view)
{
	SpinorField f, g; wrap(f, a); set_view(f, view);
	if(b) { wrap(g, b); set_view(g, view); }
	complex c(re, im);
	switch(op)
	{
		case 0: spinor_add_assign(f, g); break;
		case 1: spinor_sub_assign(f, g); break;
		case 2: spinor_mulr(f, re, g); break;
		case 3: spinor_mulc(f, c, g); break;
		case 4: spinor_mulr_assign(f, re); break;
		case 5: spinor_mulc_assign(f, c); break;
		case 6: spinor_mulr_add_assign(f, re, g); break;
		case 7: spinor_mulc_add_assign(f, c, g); break;
		case 8: spinor_mulr_sub_assign(f, re, g); break;
		case 9: spinor_mulc_sub_assign(f, c, g); break;
	}
}

/* ---- inverters (inverter.h); op: 0 Dphi, 1 Hphi, 2 Hphi_sq ---- */
int yref_cg(int op, double mass, double prec, double *x, double *b)
{
	inv_par par; SpinorField fx, fb; wrap(fx, x); wrap(fb, b);
	par.prec = prec; par.mass = mass; par.mvm = op_from_id(op);
	return cg_inverter(par, fx, fb);
}
int yref_bicgstab(int op, double mass, double prec, double *x, double *b)
{
	inv_par par; SpinorField fx, fb; wrap(fx, x); wrap(fb, b);
	par.prec = prec; par.mass = mass; par.mvm = op_from_id(op);
	return bicgstab_inverter(par, fx, fb);
}
int yref_minres(int op, double mass, double prec, double *x, double *b)
{
	inv_par par; SpinorField fx, fb; wrap(fx, x); wrap(fb, b);
	par.prec = prec; par.mass = mass; par.mvm = op_from_id(op);
	return minres_inverter(par, fx, fb);
}
int yref_auto_inverter(int op, double mass, double prec, double *x, double *b)
{
	inv_par par; SpinorField fx, fb; wrap(fx, x); wrap(fb, b);
	par.prec = prec; par.mass = mass; par.mvm = op_from_id(op);
	return auto_inverter(par, fx, fb);
}
/* xs: num consecutive spinor fields */
int yref_cg_mshift(int op, double mass, double prec, int num, double *shifts, double *xs, double *b)
{
	inv_par par; SpinorField fb; wrap(fb, b);
	SpinorField *fx = new SpinorField[num];
	long stride = (long)outer.vol4 * (sizeof(Spinor)/sizeof(double));
	for(int n = 0; n < num; n++) wrap(fx[n], xs + n*stride);
	par.prec = prec; par.mass = mass; par.mvm = op_from_id(op); par.num = num; par.shift = shifts;
	int it = cg_mshift(par, fx, fb);
	delete[] fx;
	return it;
}

/* rational_find + rational_calc (rational.cpp:68-166); meta out: order, a0, poles[], residues[] */
void yref_rational(int n, int d, double rprec, double emin, double emax, int op, double mass,
                   double prec, double *x, double *b, double *meta)
{
	rational_app app;
	rational_find(app, n, d, rprec, emin, emax);
	SpinorField fx, fb; wrap(fx, x); wrap(fb, b);
	rational_calc(app, op_from_id(op), mass, prec, fx, fb);
	meta[0] = app.order;
	meta[1] = app.a0;
	for(int i = 0; i < app.order; i++)
	{
		meta[2+i] = app.pole[i];
		meta[2+48+i] = app.residue[i];
	}
}

/* ---- forces (forces.h); momenta live in afield_momenta ---- */
void yref_zero_momenta(void)
{
	suNa zero;
	for(int id = 0; id < 4*outer.vol4; id++) afield_momenta[id] = zero;
}
void yref_get_momenta(double *out) { memcpy(out, afield_momenta, sizeof(suNa)*4*outer.vol4); }
void yref_set_momenta(const double *in) { memcpy(afield_momenta, in, sizeof(suNa)*4*outer.vol4); }
void yref_begin_fermion_force(void) { begin_fermion_force(); }
void yref_end_fermion_force(double dt) { end_fermion_force(dt); }
void yref_wilson_fermion_force(double dt, double mass, double residue, double *lhs, double *rhs)
{
	SpinorField l, r; wrap(l, lhs); wrap(r, rhs);
	wilson_fermion_force(dt, mass, residue, l, r);
}
void yref_wilson_fermion_force_q(double dt, double mass, double residue, double *rhs)
{
	SpinorField r; wrap(r, rhs);
	wilson_fermion_force_q(dt, mass, residue, r);
}
void yref_clover_fermion_force(double residue, double *lhs, double *rhs)
{
#ifdef CLOVER_TERM
	SpinorField l, r; wrap(l, lhs); wrap(r, rhs);
	clover_fermion_force(residue, l, r);
#endif
}
void yref_clover_logdet_force(double mass, double residue) { clover_logdet_force(mass, residue); }
void yref_wilson_gauge_force(double dt, double beta) { wilson_gauge_force(dt, beta); }
void yref_improved_gauge_force(double dt, double beta, double c0, double c1) { improved_gauge_force(dt, beta, c0, c1); }
double yref_avr_wilson(int h, int w) { return avr_wilson(h, w); }

/* ---- molecular-dynamics support (update.h) ---- */
void yref_update_links(double eps) { update_links(eps); }
void yref_reunitarize(void) { reunitarize(); }
void yref_represent_gauge_field(void) { represent_gauge_field(); }
double yref_hamiltonian(void) { return hamiltonian(); }     /* no monomials: the momentum part */

/* ---- gauge configuration files (gaugefield.cpp:44-179, hirep.cpp:56-212) ---- */
/* ---- propagators and mesons (observables/propagator.cpp, observables/mesons.cpp) ---- */
void yref_point_source(int n, int tau, double *out) { SpinorField f; wrap(f, out); create_point_source(n, tau, f); }
void yref_semwall_source(int n, int tau, double *io) { SpinorField f; wrap(f, io); create_semwall_source(n, tau, f); }
void yref_calc_propagator(double m, double prec, double *dst, double *src)
{
	SpinorField d, s;
	wrap(d, dst);
	wrap(s, src);
	calc_propagator(m, prec, d, s);
}
/* the generator's state through the reference's rand_store / rand_load (random.cpp:36-46);
 * rand_init may run only once per process (it registers an atexit free each time) */
int yref_rand_store(void *buf) { return rand_store(buf); }
void yref_rand_load(void *buf, int sz) { rand_load(buf, sz); }
void yref_rand_uniform(int n, double *out) { for(int i = 0; i < n; i++) out[i] = rand_uniform(); }
/* meson_init + meson_measure; the log (which carries the correlators) goes to `log`.
 * logger_init registers an atexit fclose each time, so the first call's file is kept for
 * the rest of the process and later calls append to it. */
void yref_mesons(double mass, double prec, int hits, int method, const char *log)
{
	static int logger_on = 0;
	if(!logger_on)
	{
		logger_init(log, INFO);
		logger_on = 1;
	}
	meson_init(mass, prec, hits, method);
	meson_measure();
	fflush(NULL);
}

/* ---- Wilson and fermion flow (observables/wilsonflow.cpp, observables/fermionflow.cpp) ---- */
void yref_wf_init(void) { wf_init(); }
void yref_wf_zeta(double a) { wf_zeta(a); }
void yref_wf_update(double v) { wf_update(v); }
void yref_wf_iterate(double eps) { wf_iterate(eps); }
void yref_wf_observables(double *out) { out[0] = wf_e_plaq(); out[1] = wf_e_sym(); out[2] = wf_charge(); }
/* the flowed fields wrap the caller's buffers, which must outlive the iterate calls */
static SpinorField wf_fields[32];
void yref_wf_fermion_init(double **ptrs, int n)
{
	for(int i = 0; i < n; i++) wrap(wf_fields[i], ptrs[i]);
	wf_fermion_init(wf_fields, n);
}
void yref_wf_fermion_iterate(double eps) { wf_fermion_iterate(eps); }

void yref_gauge_save(const char *path) { gauge_field_save(path); }
void yref_gauge_load(const char *path) { gauge_field_load(path); }
void yref_gauge_save_hirep(const char *path) { gauge_field_save_hirep(path); }
void yref_gauge_load_hirep(const char *path) { gauge_field_load_hirep(path); }

/* ---- chronological initial guess (mre.h) ---- */
static mre_par mre_state;
void yref_mre_init(int max, int op, double mass) { mre_init(mre_state, max, op_from_id(op), mass); }
void yref_mre_store(double *f) { SpinorField s; wrap(s, f); mre_store(mre_state, s); }
void yref_mre_guess(double *dst, double *src) { SpinorField d, s; wrap(d, dst); wrap(s, src); mre_guess(mre_state, d, s); }
void yref_mre_reset(void) { mre_reset(mre_state); }

/* ---- the reference's own self-checks (checks/check.cpp:4-26) ---- */
int yref_check_group(void) { return check_group(); }
int yref_check_dirac(void) { return check_dirac(); }
int yref_check_inverters(void) { return check_inverters(); }

double yref_timestamp(void) { return timestamp(); }

/* ---- HMC with monomials (update.cpp:41-339, integrator.cpp, monomials/*.cpp) ----
 * yref_hmc_init reads [integrator]/[monomial] sections (the cfg format of programs/hmc.cpp)
 * and calls hmc_init(); the other calls replay the steps of update() one by one, so that a
 * test can read H before and after the integration, integrate backwards, and count MVMs. */
int yref_hmc_init(const char *cfg_text)
{
	char path[] = "/tmp/yahmc_oracle_hmcXXXXXX";
	int fd = mkstemp(path);
	if(fd < 0) return -2;
	FILE *fp = fdopen(fd, "w");
	fputs(cfg_text, fp);
	fclose(fp);
	var_init(path);
	remove(path);
	hmc_init();
	return 0;
}

void yref_hmc_reset(void) { reset_variables(); }          /* momenta + pseudo-fermions */
double yref_hmc_hamiltonian(void) { return hamiltonian(); }

/* ipar->integrator(length, ipar) of update() (update.cpp:297-299), with the integrator chain
 * given level by level from the outermost: type 0 o2lf, 1 o2mn, 2 o4mn */
void yref_hmc_integrate(double length, int nlev, const int *types, const int *steps)
{
	int_par *chain = new int_par[nlev];
	for(int i = 0; i < nlev; i++)
	{
		chain[i].level = nlev - 1 - i;
		chain[i].steps = steps[i];
		chain[i].integrator = types[i] == 0 ? &o2lf_multilevel : (types[i] == 1 ? &o2mn_multilevel : &o4mn_multilevel);
		chain[i].next = (i + 1 < nlev) ? &chain[i + 1] : 0;
	}
	chain[0].integrator(length, &chain[0]);
	delete[] chain;
}

/* one whole trajectory through update() (update.cpp:281-339), Metropolis step included */
void yref_hmc_update(double length) { update(length); }
void yref_hmc_counters(int *out) { out[0] = num_cnfg; out[1] = num_accept; }
void yref_gauge_backup(void) { gauge_field_backup(); }
void yref_gauge_restore(void) { gauge_field_restore(); }

/* A rational approximation of a chosen order from the reference's table (include/approx.h):
 * among the entries for x^(|n|/|d|) of that order, the one with the widest interval; then the
 * steps of rational_find after its choice (rational.cpp:101-131): roots and poles swapped for
 * a positive power, rescale(max), the partial-fraction residues.  out: order, a0, prec, min,
 * max, then order poles and order residues.  Returns -1 if the table has no such entry. */
int yref_rational_order(int n, int d, int order, double max, double *out)
{
	int sz = sizeof(appdb)/sizeof(double);
	int bi = -1, to = 0;
	double best = 0;
	for(int i = 0; i < sz; i += 7+2*to)
	{
		int tn = appdb[i+0], td = appdb[i+1];
		to = appdb[i+2];
		double ratio = appdb[i+4] / appdb[i+5];
		if(tn == abs(n) && td == abs(d) && to == order && (bi < 0 || ratio < best))
		{
			bi = i;
			best = ratio;
		}
	}
	if(bi < 0) return -1;
	rational_app data;
	data.n = n;
	data.d = d;
	data.order = order;
	data.prec = appdb[bi+3];
	data.min = appdb[bi+4];
	data.max = appdb[bi+5];
	data.a0 = appdb[bi+6];
	for(int i = 0; i < order; i++)
	{
		data.root[i] = appdb[7+bi+i];
		data.pole[i] = appdb[7+bi+order+i];
	}
	if(d*n > 0)
	{
		for(int i = 0; i < order; i++)
		{
			double r = data.root[i];
			data.root[i] = data.pole[i];
			data.pole[i] = r;
		}
		data.a0 = 1.0 / data.a0;
	}
	rescale(data, max);
	for(int i = 0; i < order; i++) data.residue[i] = residue(data, i);
	out[0] = order;
	out[1] = data.a0;
	out[2] = data.prec;
	out[3] = data.min;
	out[4] = data.max;
	for(int i = 0; i < order; i++)
	{
		out[5+i] = data.pole[i];
		out[5+order+i] = data.residue[i];
	}
	return 0;
}

}
