/*
 * yahmc_gpu_shim.cpp -- YaHMC's own fermion call surface over the B200 engine.
 *
 * A YaHMC build replaces eight of its library files with this one and links the engine
 * (include/yahmc_gpu.h, libyahmc_b200.so):
 *
 *   library/dirac.cpp     Dphi_oe/eo/ee/oo/oo_inv, Dphi, Hphi, Hphi_sq, mvm_get/reset
 *   library/linalg.cpp    spinor_allocate and every spinor_* function, the view selectors
 *   library/cg.cpp        cg_inverter, cg_mshift
 *   library/bicgstab.cpp  bicgstab_inverter
 *   library/minres.cpp    minres_inverter
 *   library/inverter.cpp  auto_inverter
 *   library/forces.cpp    fermion and gauge forces, begin/end_fermion_force
 *   library/clover.cpp    clover term, LDL, logdet, clover force, clover_init
 *
 * Every signature is the one in the reference's dirac.h, linalg.h, inverter.h, forces.h and
 * clover.h, so the monomials, integrators, update(), MRE, rational_calc, evlimits, the
 * observables and the --run-checks suite compile and run unchanged on top of it.  This file
 * is compiled with the reference's headers and its compile-time switches (-DNC, -DREPR_*,
 * -DBC_*, -DCLOVER_TERM, -DUPDATE_EO).
 *
 * Where the data lives
 *  - Spinor fields.  SpinorField (spinorfield.h) is unchanged: its destructor still calls
 *    delete[] on ptr, so ptr stays a host array of outer.vol4 Spinors allocated with new[].
 *    Each such array has a device twin, found by its address.  A field allocated here by
 *    spinor_allocate lives on the device: operations read and write the twin and the host
 *    array is left alone.  A host array this file did not allocate (a caller's own buffer)
 *    is host data: it is uploaded before and downloaded after every operation that touches
 *    it.  Setting YAHMC_GPU_HOST_MIRROR=1 treats every field that way, for callers that read
 *    or write Spinors through operator[] between operations (checks/dirac.cpp's covariance
 *    check, the observables' source and contraction code).
 *  - Gauge field.  gfield_fund stays the host master copy, as update.cpp changes it there.
 *    represent_gauge_field() (repr.cpp, unchanged) ends in compute_clover_term(), which
 *    uploads the links; the engine represents them, rebuilds the clover term and applies
 *    the antiperiodic sign.  The gauge forces upload the fundamental links alone, since
 *    update_links changes them on the host between two represent_gauge_field calls.
 *  - Momenta.  afield_momenta stays the host master copy (reset_variables, update_links and
 *    hamiltonian() read it there).  begin_fermion_force uploads it, the fermion forces of
 *    the level accumulate on the device, end_fermion_force downloads it; a force called
 *    outside that bracket uploads and downloads around itself.
 *  - Random numbers are drawn on the host by the reference's own generator (spinor_random
 *    fills the host array with Spinor::randomize, then uploads), so a GPU build and a CPU
 *    build started from the same seed consume the same random stream.
 *
 * Run-time options (environment)
 *  - YAHMC_GPU_DEVICE=n          CUDA device of this process (one process per GPU)
 *  - YAHMC_GPU_HOST_MIRROR=1     keep every spinor field's host array in step (see above)
 *  - YAHMC_GPU_SOLVER=mixed      solves of Hphi_sq (cg_inverter, auto_inverter) use the
 *                                mixed-precision CG, which stops on the true FP64 residual
 *                                |b - A x|^2 < prec |b|^2; default: the reference's algorithms
 *
 * Errors: a failing engine call is reported through lprintf(CRITICAL), which ends the
 * program as the reference's own errors do (logger.cpp:53-56).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

#include <yahmc_gpu.h>

/* reference headers last: include/gaugefield.h defines a macro named link */
#include <global.h>
#include <linalg.h>
#include <dirac.h>
#include <inverter.h>
#include <forces.h>
#include <clover.h>
#include <bcs.h>
#include <repr.h>
#include <logger.h>
#include <memory.h>
#include <timing.h>

/* ---- the reference's clover globals (clover.h:35-37) ---------------------------------
 * Kept as host arrays so that code reading them still finds storage; the engine owns the
 * device copies.  cl_ldl receives the factors when compute_ldl_decomp is called. */
suNf *cl_force = 0;
suNf *cl_term = 0;
ldl_t *cl_ldl = 0;

namespace {

struct Twin {
	double *dev;
	bool owned;       // allocated by spinor_allocate: the device copy is the field
};

yg_lattice *g_lat = 0;
yg_info g_info;
double g_csw = 0;
bool g_mirror = false;
bool g_mixed = false;
bool g_mom_on_device = false;
std::unordered_map<const void*, Twin> g_twins;

void check(int rc, const char *what)
{
	if(rc != YG_OK)
	{
		lprintf("GPU", CRITICAL, "%s failed: %s", what, yg_last_error());
	}
}

int bc_id()
{
#if defined(BC_ANTIPERIODIC)
	return YG_BC_ANTIPERIODIC;
#elif defined(BC_OPEN)
	return YG_BC_OPEN;
#elif defined(BC_SF)
	return YG_BC_SF;
#else
	return YG_BC_PERIODIC;
#endif
}

/* The device lattice, created at the first call that needs it (after geometry_init,
 * bcs_init and clover_init, as in programs/hmc.cpp:94-117). */
yg_lattice *lat()
{
	if(g_lat)
	{
		return g_lat;
	}

	const char *env = getenv("YAHMC_GPU_DEVICE");
	if(env)
	{
		check(yg_set_device(atoi(env)), "yg_set_device");
	}
	env = getenv("YAHMC_GPU_HOST_MIRROR");
	g_mirror = env && atoi(env) != 0;
	env = getenv("YAHMC_GPU_SOLVER");
	g_mixed = env && strcmp(env, "mixed") == 0;

	yg_params p;
	p.dims[0] = global.dim_t;
	p.dims[1] = global.dim_x;
	p.dims[2] = global.dim_y;
	p.dims[3] = global.dim_z;
	p.nc = NC;
	p.repr = REPR_ID;
	p.bc = bc_id();
#ifdef CLOVER_TERM
	p.clover = 1;
#else
	p.clover = 0;
#endif
#ifdef UPDATE_EO
	p.eo = 1;
#else
	p.eo = 0;
#endif
	p.csw = g_csw;
	p.cf = (p.bc == YG_BC_OPEN || p.bc == YG_BC_SF) ? bcs.cf : 1.0;
	check(yg_lattice_create(&p, &g_lat), "yg_lattice_create");
	check(yg_lattice_query(g_lat, &g_info), "yg_lattice_query");

	// the host master copies travel often: page-lock them once
	if(gfield_fund)
	{
		check(yg_host_register(gfield_fund, sizeof(suNg)*4*outer.vol4), "yg_host_register(gfield_fund)");
	}
	if(afield_momenta)
	{
		check(yg_host_register(afield_momenta, sizeof(suNa)*4*outer.vol4), "yg_host_register(afield_momenta)");
	}

	lprintf("GPU", INFO, "B200 engine: %dx%dx%dx%d, %s%s", p.dims[0], p.dims[1], p.dims[2], p.dims[3],
	        g_mirror ? "host mirror on" : "fields device-resident",
	        g_mixed ? ", mixed-precision CG for Hphi_sq" : "");
	return g_lat;
}

Twin &twin(SpinorField &sf)
{
	if(sf.ptr == 0)
	{
		lprintf("GPU", CRITICAL, "spinor field used before spinor_allocate");
	}
	auto it = g_twins.find(sf.ptr);
	if(it != g_twins.end())
	{
		return it->second;
	}
	Twin t;
	check(yg_field_alloc(lat(), &t.dev), "yg_field_alloc");
	t.owned = false;
	return g_twins.emplace(sf.ptr, t).first->second;
}

bool host_side(const Twin &t)
{
	return g_mirror || !t.owned;
}

/* The fields of one operation: host-side fields are uploaded when first named and
 * downloaded when the operation ends (every field an operation names may be written:
 * Dphi writes into its source, the fermion forces into both arguments). */
class Fields {
public:
	double *operator()(SpinorField &sf)
	{
		Twin &t = twin(sf);
		for(auto &a : args)
		{
			if(a.first == &sf || a.first->ptr == sf.ptr)
			{
				return t.dev;
			}
		}
		args.push_back(std::make_pair(&sf, &t));
		if(host_side(t))
		{
			check(yg_field_upload(lat(), t.dev, (const double*)sf.ptr), "yg_field_upload");
		}
		return t.dev;
	}

	~Fields()
	{
		for(auto &a : args)
		{
			if(host_side(*a.second))
			{
				check(yg_field_download(lat(), (double*)a.first->ptr, a.second->dev), "yg_field_download");
			}
		}
	}

private:
	std::vector<std::pair<SpinorField*, Twin*> > args;
};

int view(SpinorField &sf)
{
	if(sf.sites == local.vol4)
	{
		return YG_VIEW_FULL;
	}
	return sf.offset ? YG_VIEW_ODD : YG_VIEW_EVEN;
}

void match(SpinorField &a, SpinorField &b)
{
	if(a.sites != b.sites)
	{
		lprintf("LINALG", CRITICAL, "Spinors do not match");
	}
}

/* The momenta on the device for the duration of one force call, unless a fermion-force
 * bracket already holds them there. */
class Momenta {
public:
	Momenta() : own(!g_mom_on_device)
	{
		if(own)
		{
			check(yg_momenta_upload(lat(), (const double*)afield_momenta), "yg_momenta_upload");
		}
	}
	~Momenta()
	{
		if(own)
		{
			check(yg_momenta_download(lat(), (double*)afield_momenta), "yg_momenta_download");
		}
	}
private:
	bool own;
};

int op_id(mvm_operator f, const char *who)
{
	if(f == Hphi_sq) return YG_OP_HPHI_SQ;
	if(f == Hphi) return YG_OP_HPHI;
	if(f == Dphi) return YG_OP_DPHI;
	lprintf("INVERTER", CRITICAL, "%s: no MVM operator specified", who);
	return -1;
}

yg_inv_par inv(inv_par &par, const char *who)
{
	yg_inv_par p;
	p.op = op_id(par.mvm, who);
	p.mass = par.mass;
	p.prec = par.prec;
	p.log = 0;
	p.maxiter = 0;
	return p;
}

/* the mixed-precision CG on Hphi_sq; returns its inner iteration count */
int cg_mixed(inv_par &par, SpinorField &x, SpinorField &b, const char *who)
{
	yg_inv_par p = inv(par, who);
	yg_solve_stats st;
	Fields f;
	double *dx = f(x), *db = f(b);
	const int rc = yg_cg_mixed(lat(), &p, dx, db, &st);
	if(rc == YG_STALL)
	{
		// the true residual could not be brought below prec (an ill-conditioned system whose
		// FP64 rounding floor lies above it); x is the FP64 CG's solution, which met prec on
		// its recursive residual, which is all YaHMC's own cg_inverter (cg.cpp:186) asks for
		lprintf("INVERTER", NOTICE, "%s (mixed CG): true residual %1.4e above prec %1.1e, kept the FP64 CG's solution",
		        who, st.true_residual, par.prec);
	}
	else
	{
		check(rc, "yg_cg_mixed");
	}
	if(par.log)
	{
		lprintf("INVERTER", NOTICE, "%s (mixed CG): iterations = %d, precision = %1.4e, reliable updates = %d%s",
		        who, st.iterations, st.true_residual, st.reliable_updates, st.fallback ? ", FP64 fallback" : "");
	}
	return st.iterations;
}

}  // namespace

/* ---- dirac.h (dirac.cpp:9-781) -------------------------------------------------------- */
int mvm_get()
{
	return yg_mvm_get(lat());
}

void mvm_reset()
{
	yg_mvm_reset(lat());
}

void Dphi_oe(SpinorField &dptr, SpinorField &sptr)
{
	timing_start(tm_hopping_term);
	Fields f;
	double *d = f(dptr), *s = f(sptr);
	check(yg_Dphi_oe(lat(), d, s), "yg_Dphi_oe");
	timing_end(tm_hopping_term);
}

void Dphi_eo(SpinorField &dptr, SpinorField &sptr)
{
	timing_start(tm_hopping_term);
	Fields f;
	double *d = f(dptr), *s = f(sptr);
	check(yg_Dphi_eo(lat(), d, s), "yg_Dphi_eo");
	timing_end(tm_hopping_term);
}

void Dphi_ee(double mass, SpinorField &dptr, SpinorField &sptr)
{
	timing_start(tm_clover_term);
	Fields f;
	double *d = f(dptr), *s = f(sptr);
	check(yg_Dphi_ee(lat(), mass, d, s), "yg_Dphi_ee");
	timing_end(tm_clover_term);
}

void Dphi_oo(double mass, SpinorField &dptr, SpinorField &sptr)
{
	timing_start(tm_clover_term);
	Fields f;
	double *d = f(dptr), *s = f(sptr);
	check(yg_Dphi_oo(lat(), mass, d, s), "yg_Dphi_oo");
	timing_end(tm_clover_term);
}

void Dphi_oo_inv(double mass, SpinorField &dptr, SpinorField &sptr)
{
	timing_start(tm_clover_term);
	Fields f;
	double *d = f(dptr), *s = f(sptr);
	check(yg_Dphi_oo_inv(lat(), mass, d, s), "yg_Dphi_oo_inv");
	timing_end(tm_clover_term);
}

void Dphi(double mass, SpinorField &dptr, SpinorField &sptr)
{
	timing_start(tm_hopping_term);
	Fields f;
	double *d = f(dptr), *s = f(sptr);
	check(yg_Dphi(lat(), mass, d, s), "yg_Dphi");
	timing_end(tm_hopping_term);
}

void Hphi(double mass, SpinorField &dptr, SpinorField &sptr)
{
	timing_start(tm_hopping_term);
	Fields f;
	double *d = f(dptr), *s = f(sptr);
	check(yg_Hphi(lat(), mass, d, s), "yg_Hphi");
	timing_end(tm_hopping_term);
}

void Hphi_sq(double mass, SpinorField &dptr, SpinorField &sptr)
{
	timing_start(tm_hopping_term);
	Fields f;
	double *d = f(dptr), *s = f(sptr);
	check(yg_Hphi_sq(lat(), mass, d, s), "yg_Hphi_sq");
	timing_end(tm_hopping_term);
}

/* ---- linalg.h (linalg.cpp:10-329) ----------------------------------------------------- */
void spinor_allocate(SpinorField &sf)
{
	if(sf.allocated)
	{
		return;
	}
	sf.ptr = new Spinor[outer.vol4];
	sf.allocated = true;
	spinor_type_default(sf);
	bool reused = g_twins.count(sf.ptr) != 0;
	Twin &t = twin(sf);
	if(reused)
	{
		// a new array at the address of a freed one (rational_calc allocates and frees its
		// fields per call): start from zero, as new Spinor[] does
		check(yg_spinor_zero(lat(), t.dev), "yg_spinor_zero");
	}
	t.owned = true;
}

void spinor_zero(SpinorField &sf)
{
	timing_start(tm_linalg);
	Fields f;
	check(yg_spinor_zero(lat(), f(sf)), "yg_spinor_zero");
	timing_end(tm_linalg);
}

/* The reference's draw: Spinor::randomize for every site of the view in order, then the
 * spinor boundary conditions (linalg.cpp:42-53), on the host array; then the field goes up.
 * A device-resident field is brought down first so that the sites outside the view keep
 * their values. */
void spinor_random(SpinorField &sf)
{
	timing_start(tm_linalg);
	Twin &t = twin(sf);
	if(!host_side(t))
	{
		check(yg_field_download(lat(), (double*)sf.ptr, t.dev), "yg_field_download");
	}
	spinor_for(id,sf)
	{
		sf[id].randomize();
	}
	apply_bcs_on_spinor_field(sf);
	check(yg_field_upload(lat(), t.dev, (const double*)sf.ptr), "yg_field_upload");
	timing_end(tm_linalg);
}

double spinor_sqnorm(SpinorField &sf)
{
	double r = 0;
	timing_start(tm_linalg);
	Fields f;
	check(yg_spinor_sqnorm(lat(), f(sf), view(sf), &r), "yg_spinor_sqnorm");
	timing_end(tm_linalg);
	return r;
}

void spinor_copy(SpinorField &lhs, SpinorField &rhs)
{
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_copy(lat(), a, b), "yg_spinor_copy");
	timing_end(tm_linalg);
}

void spinor_g5(SpinorField &sf)
{
	timing_start(tm_linalg);
	Fields f;
	check(yg_spinor_g5(lat(), f(sf), view(sf)), "yg_spinor_g5");
	timing_end(tm_linalg);
}

void spinor_add_assign(SpinorField &lhs, SpinorField &rhs)
{
	match(lhs, rhs);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_add_assign(lat(), a, b, view(lhs)), "yg_spinor_add_assign");
	timing_end(tm_linalg);
}

void spinor_sub_assign(SpinorField &lhs, SpinorField &rhs)
{
	match(lhs, rhs);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_sub_assign(lat(), a, b, view(lhs)), "yg_spinor_sub_assign");
	timing_end(tm_linalg);
}

void spinor_mulr(SpinorField &lhs, double v, SpinorField &rhs)
{
	match(lhs, rhs);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_mulr(lat(), a, v, b, view(lhs)), "yg_spinor_mulr");
	timing_end(tm_linalg);
}

void spinor_mulc(SpinorField &lhs, complex v, SpinorField &rhs)
{
	match(lhs, rhs);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_mulc(lat(), a, v.re, v.im, b, view(lhs)), "yg_spinor_mulc");
	timing_end(tm_linalg);
}

void spinor_mulr_assign(SpinorField &lhs, double v)
{
	timing_start(tm_linalg);
	Fields f;
	check(yg_spinor_mulr_assign(lat(), f(lhs), v, view(lhs)), "yg_spinor_mulr_assign");
	timing_end(tm_linalg);
}

void spinor_mulc_assign(SpinorField &lhs, complex v)
{
	timing_start(tm_linalg);
	Fields f;
	check(yg_spinor_mulc_assign(lat(), f(lhs), v.re, v.im, view(lhs)), "yg_spinor_mulc_assign");
	timing_end(tm_linalg);
}

void spinor_mulr_add_assign(SpinorField &lhs, double v, SpinorField &rhs)
{
	match(lhs, rhs);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_mulr_add_assign(lat(), a, v, b, view(lhs)), "yg_spinor_mulr_add_assign");
	timing_end(tm_linalg);
}

void spinor_mulc_add_assign(SpinorField &lhs, complex v, SpinorField &rhs)
{
	match(lhs, rhs);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_mulc_add_assign(lat(), a, v.re, v.im, b, view(lhs)), "yg_spinor_mulc_add_assign");
	timing_end(tm_linalg);
}

void spinor_mulr_sub_assign(SpinorField &lhs, double v, SpinorField &rhs)
{
	match(lhs, rhs);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_mulr_sub_assign(lat(), a, v, b, view(lhs)), "yg_spinor_mulr_sub_assign");
	timing_end(tm_linalg);
}

void spinor_mulc_sub_assign(SpinorField &lhs, complex v, SpinorField &rhs)
{
	match(lhs, rhs);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_spinor_mulc_sub_assign(lat(), a, v.re, v.im, b, view(lhs)), "yg_spinor_mulc_sub_assign");
	timing_end(tm_linalg);
}

complex spinor_product(SpinorField &sf_a, SpinorField &sf_b)
{
	double r[2] = {0, 0};
	match(sf_a, sf_b);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(sf_a), *b = f(sf_b);
	check(yg_spinor_product(lat(), a, b, view(sf_a), r), "yg_spinor_product");
	timing_end(tm_linalg);
	return complex(r[0], r[1]);
}

double spinor_product_re(SpinorField &sf_a, SpinorField &sf_b)
{
	double r = 0;
	match(sf_a, sf_b);
	timing_start(tm_linalg);
	Fields f;
	double *a = f(sf_a), *b = f(sf_b);
	check(yg_spinor_product_re(lat(), a, b, view(sf_a), &r), "yg_spinor_product_re");
	timing_end(tm_linalg);
	return r;
}

/* views: the same site ranges as linalg.cpp:272-329 */
void spinor_select_even(SpinorField &sf)
{
	sf.offset = 0;
	sf.sites = (local.vol4 / 2);
}

void spinor_select_odd(SpinorField &sf)
{
	sf.offset = (local.vol4 / 2);
	sf.sites = (local.vol4 / 2);
}

void spinor_select_full(SpinorField &sf)
{
	sf.offset = 0;
	sf.sites = local.vol4;
}

void spinor_select_default(SpinorField &sf)
{
	sf.offset = sf.default_offset;
	sf.sites = sf.default_sites;
}

void spinor_type_even(SpinorField &sf)
{
	sf.default_offset = 0;
	sf.default_sites = (local.vol4 / 2);
	spinor_select_default(sf);
}

void spinor_type_odd(SpinorField &sf)
{
	sf.default_offset = (local.vol4 / 2);
	sf.default_sites = (local.vol4 / 2);
	spinor_select_default(sf);
}

void spinor_type_full(SpinorField &sf)
{
	sf.default_offset = 0;
	sf.default_sites = local.vol4;
	spinor_select_default(sf);
}

void spinor_type_default(SpinorField &sf)
{
#ifdef UPDATE_EO
	spinor_type_even(sf);
#else
	spinor_type_full(sf);
#endif
}

/* ---- inverter.h (cg.cpp, bicgstab.cpp, minres.cpp, inverter.cpp) ----------------------- */
int cg_inverter(inv_par &par, SpinorField &dptr, SpinorField &sptr)
{
	if(g_mixed && par.mvm == Hphi_sq)
	{
		return cg_mixed(par, dptr, sptr, "cg");
	}
	yg_inv_par p = inv(par, "cg");
	int it = 0;
	Fields f;
	double *x = f(dptr), *b = f(sptr);
	check(yg_cg_inverter(lat(), &p, x, b, &it), "yg_cg_inverter");
	if(par.log)
	{
		lprintf("INVERTER", NOTICE, "cg: iterations = %d", it);
	}
	return it;
}

int cg_mshift(inv_par &par, SpinorField *dptr, SpinorField &sptr)
{
	yg_inv_par p = inv(par, "cg_mshift");
	int it = 0;
	Fields f;
	std::vector<double*> xs(par.num);
	for(int n = 0; n < par.num; n++)
	{
		xs[n] = f(dptr[n]);
	}
	double *b = f(sptr);
	check(yg_cg_mshift(lat(), &p, par.num, par.shift, xs.data(), b, &it), "yg_cg_mshift");
	if(par.log)
	{
		lprintf("INVERTER", NOTICE, "cg_mshift: iterations = %d", it);
	}
	return it;
}

int bicgstab_inverter(inv_par &par, SpinorField &dptr, SpinorField &sptr)
{
	yg_inv_par p = inv(par, "bicgstab");
	int it = 0;
	Fields f;
	double *x = f(dptr), *b = f(sptr);
	check(yg_bicgstab_inverter(lat(), &p, x, b, &it), "yg_bicgstab_inverter");
	if(par.log)
	{
		lprintf("INVERTER", NOTICE, "bicgstab: iterations = %d", it);
	}
	return it;
}

int minres_inverter(inv_par &par, SpinorField &dptr, SpinorField &sptr)
{
	yg_inv_par p = inv(par, "minres");
	int it = 0;
	Fields f;
	double *x = f(dptr), *b = f(sptr);
	check(yg_minres_inverter(lat(), &p, x, b, &it), "yg_minres_inverter");
	if(par.log)
	{
		lprintf("INVERTER", NOTICE, "minres: iterations = %d", it);
	}
	return it;
}

int auto_inverter(inv_par &par, SpinorField &dptr, SpinorField &sptr)
{
	if(par.num > 0)
	{
		lprintf("INVERTER", CRITICAL, "auto: no support for multishift inversion");
	}
	if(g_mixed && par.mvm == Hphi_sq)
	{
		return cg_mixed(par, dptr, sptr, "auto");
	}
	yg_inv_par p = inv(par, "auto");
	int it = 0;
	Fields f;
	double *x = f(dptr), *b = f(sptr);
	check(yg_auto_inverter(lat(), &p, x, b, &it), "yg_auto_inverter");
	return it;
}

/* ---- clover.h (clover.cpp) -------------------------------------------------------------- */
double get_csw()
{
	return g_csw;
}

void clover_init(double csw)
{
#ifdef CLOVER_TERM
	g_csw = csw;
	cl_force = suNf_allocate(6);
	cl_term = suNf_allocate(4);
	cl_ldl = ldl_allocate(1);
	lprintf("CLOVER", INFO, "Coefficient: csw = %1.4f", g_csw);
#endif
}

/* Called at the end of represent_gauge_field (repr.cpp:265-280) and nowhere else: every
 * change of the gauge field reaches the device here, with or without a clover term. */
void compute_clover_term()
{
	timing_start(tm_clover_term);
	check(yg_gauge_upload(lat(), (const double*)gfield_fund), "yg_gauge_upload");
#ifdef CLOVER_TERM
	if(g_mirror)
	{
		check(yg_clover_term_download(lat(), (double*)cl_term), "yg_clover_term_download");
	}
#endif
	timing_end(tm_clover_term);
}

/* The engine keeps its factors for the last sigma on the device and refreshes them itself;
 * here they are also brought to the host cl_ldl for code that reads it. */
void compute_ldl_decomp(double sigma)
{
#ifdef CLOVER_TERM
	check(yg_ldl_download(lat(), sigma - 4.0, (double*)cl_ldl), "yg_ldl_download");
#endif
}

double clover_logdet(double mass)
{
	double r = 0;
	timing_start(tm_clover_term);
	check(yg_clover_logdet(lat(), mass, &r), "yg_clover_logdet");
	timing_end(tm_clover_term);
	return r;
}

void compute_clover_force(double mass, double coeff)
{
	Momenta m;
	check(yg_clover_logdet_force(lat(), mass, coeff), "yg_clover_logdet_force");
}

/* ---- forces.h (forces.cpp) -------------------------------------------------------------- */
void clover_logdet_force(double mass, double residue)
{
	timing_start(tm_clover_force);
	compute_clover_force(mass, residue);
	timing_end(tm_clover_force);
}

void clover_fermion_force(double residue, SpinorField &lhs, SpinorField &rhs)
{
	timing_start(tm_clover_force);
	Momenta m;
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_clover_fermion_force(lat(), residue, a, b), "yg_clover_fermion_force");
	timing_end(tm_clover_force);
}

void wilson_fermion_force(double dt, double mass, double residue, SpinorField &lhs, SpinorField &rhs)
{
	timing_start(tm_hopping_force);
	Momenta m;
	Fields f;
	double *a = f(lhs), *b = f(rhs);
	check(yg_wilson_fermion_force(lat(), dt, mass, residue, a, b), "yg_wilson_fermion_force");
	timing_end(tm_hopping_force);
}

void wilson_fermion_force_q(double dt, double mass, double residue, SpinorField &rhs)
{
	timing_start(tm_hopping_force);
	Momenta m;
	Fields f;
	check(yg_wilson_fermion_force_q(lat(), dt, mass, residue, f(rhs)), "yg_wilson_fermion_force_q");
	timing_end(tm_hopping_force);
}

void begin_fermion_force()
{
	if(!g_mom_on_device)
	{
		check(yg_momenta_upload(lat(), (const double*)afield_momenta), "yg_momenta_upload");
		g_mom_on_device = true;
	}
	check(yg_begin_fermion_force(lat()), "yg_begin_fermion_force");
}

void end_fermion_force(double dt)
{
	timing_start(tm_clover_force);
	check(yg_end_fermion_force(lat(), dt), "yg_end_fermion_force");
	if(g_mom_on_device)
	{
		check(yg_momenta_download(lat(), (double*)afield_momenta), "yg_momenta_download");
		g_mom_on_device = false;
	}
	timing_end(tm_clover_force);
}

void wilson_gauge_force(double dt, double beta)
{
	timing_start(tm_gauge_force);
	check(yg_gauge_upload_fund(lat(), (const double*)gfield_fund), "yg_gauge_upload_fund");
	Momenta m;
	check(yg_wilson_gauge_force(lat(), dt, beta), "yg_wilson_gauge_force");
	timing_end(tm_gauge_force);
}

void improved_gauge_force(double dt, double beta, double c0, double c1)
{
	timing_start(tm_gauge_force);
	check(yg_gauge_upload_fund(lat(), (const double*)gfield_fund), "yg_gauge_upload_fund");
	Momenta m;
	check(yg_improved_gauge_force(lat(), dt, beta, c0, c1), "yg_improved_gauge_force");
	timing_end(tm_gauge_force);
}
