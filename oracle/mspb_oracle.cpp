// ORACLE — test infrastructure, not product code.
//
// A C interface over the reference's own MSPB v1 snapshot and MSPBPack archive code
// (apps/CCOptimization/MSPB_Pack.{h,cpp}), compiled from the reference tree into oracle/_ref/libccref.so. The tests
// call it as the checker of modules_b200.mspb: files written by one side must read back equal on the other, and the
// bytes either side writes for the same snapshot must be the same.
#include "MSPB_Pack.h"

#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>

namespace {

void set_err(char *err, int errlen, const std::string &msg)
{
	if (err && errlen > 0) {
		std::strncpy(err, msg.c_str(), (size_t)errlen - 1);
		err[errlen - 1] = '\0';
	}
}

}  // namespace

extern "C" {

// Write one snapshot with MSPBSnapshot::Write: d x d basis (rows = basis vectors), N particles with ids, species
// labels, relative coordinates (N x d) and radii. Returns 0, or -1 with the reference's message in err.
int ccref_mspb_write(const char *path, int d, long N, unsigned long long species_count, const double *basis,
                     const unsigned long long *ids, const unsigned *species, const double *rel, const double *radii,
                     char *err, int errlen)
{
	try {
		MSPBSnapshot s;
		s.speciesCount = species_count;
		for (int i = 0; i < d; i++) {
			GeometryVector b(d);
			for (int j = 0; j < d; j++)
				b.x[j] = basis[i * d + j];
			s.basis.push_back(b);
		}
		for (long i = 0; i < N; i++) {
			MSPBParticle p;
			p.id = ids[i];
			p.species = species[i];
			p.relative = GeometryVector(d);
			for (int e = 0; e < d; e++)
				p.relative.x[e] = rel[i * d + e];
			p.radius = radii[i];
			s.particles.push_back(p);
		}
		std::ofstream out(path, std::ios::binary);
		if (!out)
			throw std::runtime_error("cannot open output");
		s.Write(out);
		out.close();
		if (!out)
			throw std::runtime_error("cannot finish output");
		return 0;
	} catch (const std::exception &e) {
		set_err(err, errlen, e.what());
		return -1;
	}
}

// Read one snapshot file with MSPBSnapshot::Read. With basis == NULL only *d, *N and *species_count are set (to size
// the arrays of a second call). Returns 0, or -1 with the reference's message in err.
int ccref_mspb_read(const char *path, int *d, long *N, unsigned long long *species_count, double *basis,
                    unsigned long long *ids, unsigned *species, double *rel, double *radii, char *err, int errlen)
{
	try {
		std::ifstream in(path, std::ios::binary);
		if (!in)
			throw std::runtime_error("cannot open input");
		const MSPBSnapshot s = MSPBSnapshot::Read(in);
		const int dim = (int)s.basis.size();
		*d = dim;
		*N = (long)s.particles.size();
		*species_count = s.speciesCount;
		if (!basis)
			return 0;
		for (int i = 0; i < dim; i++)
			for (int j = 0; j < dim; j++)
				basis[i * dim + j] = s.basis[i].x[j];
		for (size_t i = 0; i < s.particles.size(); i++) {
			ids[i] = s.particles[i].id;
			species[i] = s.particles[i].species;
			for (int e = 0; e < dim; e++)
				rel[i * dim + e] = s.particles[i].relative.x[e];
			radii[i] = s.particles[i].radius;
		}
		return 0;
	} catch (const std::exception &e) {
		set_err(err, errlen, e.what());
		return -1;
	}
}

// MSPB_Pack(prefix).ImportFile(file). Returns 0, or -1 with the reference's message in err.
int ccref_mspbpack_import(const char *prefix, const char *file, char *err, int errlen)
{
	try {
		MSPB_Pack pack(prefix);
		pack.ImportFile(file);
		return 0;
	} catch (const std::exception &e) {
		set_err(err, errlen, e.what());
		return -1;
	}
}

// MSPB_Pack(prefix).NumConfig() into *count (the archive's framing scanned by Open). Returns 0 or -1.
int ccref_mspbpack_count(const char *prefix, long *count, char *err, int errlen)
{
	try {
		MSPB_Pack pack(prefix);
		*count = (long)pack.NumConfig();
		return 0;
	} catch (const std::exception &e) {
		set_err(err, errlen, e.what());
		return -1;
	}
}

// MSPB_Pack(prefix).ExportFile(index, file). Returns 0 or -1.
int ccref_mspbpack_export(const char *prefix, long index, const char *file, char *err, int errlen)
{
	try {
		MSPB_Pack pack(prefix);
		pack.ExportFile((size_t)index, file);
		return 0;
	} catch (const std::exception &e) {
		set_err(err, errlen, e.what());
		return -1;
	}
}

}  // extern "C"
