// jms_sli.cpp -- EMS slice files (.sli): phase gratings as written by Dr. Probe
// and read by the reference's bench driver (test/JMSBench1/prm_slice_file_info.h:
// 60-150, prm_slice_file_info.cpp load_ems_header / save_ems_header,
// prm_slice.cpp load_ems_data).
//
// Layout: an 8192-byte header, then nvar complex64 gratings [nvar][ny][nx]
// at the data offset.  Header fields used (byte offsets): nx 0x0000, ny
// 0x0004, title 0x004C (40 chars), extended header version 0x0074, number of
// variants 0x0078 (versions 2010112301, 2012071101, 2020052801; else 1),
// content type 0x0080 (0 grating, 1 potential), alternative data offset
// 0x0088 and atom-table offset 0x008C (versions 2012071101, 2020052801),
// slice thickness 0x1034, beam energy 0x1040, slice size x 0x1044 and
// y 0x1048 (float, nm / keV).  A first word outside [0, 16384] marks a file
// of the other byte order; its fields and data are swapped on input.
#include "../../include/jms_b200.h"
#include "jms_host.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {
constexpr long kPosNx = 0x0000, kPosNy = 0x0004, kPosTitle = 0x004C, kPosVer = 0x0074, kPosNvar = 0x0078;
constexpr long kPosContent = 0x0080, kPosAltOffset = 0x0088, kPosTabOffset = 0x008C;
constexpr long kPosThick = 0x1034, kPosEkv = 0x1040, kPosSx = 0x1044, kPosSy = 0x1048;
constexpr long kPosTab = 0x1100, kPosData = 0x2000;
constexpr uint32_t kVerWrite = 2020052801u;

uint32_t bswap32(uint32_t v)
{
	return (v >> 24) | ((v >> 8) & 0xFF00u) | ((v << 8) & 0xFF0000u) | (v << 24);
}

struct Reader {
	std::FILE* f = nullptr;
	bool swap = false;
	~Reader() { if (f) std::fclose(f); }
	bool u32(long pos, uint32_t* v)
	{
		if (std::fseek(f, pos, SEEK_SET) != 0 || std::fread(v, 4, 1, f) != 1) return false;
		if (swap) *v = bswap32(*v);
		return true;
	}
	bool f32(long pos, float* v)
	{
		uint32_t u;
		if (!u32(pos, &u)) return false;
		std::memcpy(v, &u, 4);
		return true;
	}
};

int read_header(Reader& R, const char* path, JMSSliHeader* h)
{
	R.f = std::fopen(path, "rb");
	if (!R.f) return 2;
	int32_t first = 0;
	if (std::fread(&first, 4, 1, R.f) != 1) return 3;
	R.swap = (first < 0 || first > 16384);
	std::memset(h, 0, sizeof(*h));
	uint32_t u = 0;
	if (!R.u32(kPosNx, &u)) return 3;
	h->nx = (int)u;
	if (!R.u32(kPosNy, &u)) return 3;
	h->ny = (int)u;
	if (std::fseek(R.f, kPosTitle, SEEK_SET) != 0 || std::fread(h->title, 1, 40, R.f) != 40) return 3;
	h->title[40] = '\0';
	if (!R.u32(kPosVer, &u)) return 3;
	h->version = u;
	if (!R.u32(kPosContent, &u)) return 3;
	h->content = (int)u;
	h->nvar = 1;
	h->data_offset = kPosData;
	h->table_offset = kPosTab;
	if (h->version == 2010112301u || h->version == 2012071101u || h->version == 2020052801u) {
		if (!R.u32(kPosNvar, &u)) return 3;
		h->nvar = (int)u;
		if (h->version != 2010112301u) {
			if (!R.u32(kPosAltOffset, &u)) return 3;
			h->data_offset = u;
			if (!R.u32(kPosTabOffset, &u)) return 3;
			h->table_offset = u;
		}
	}
	if (!R.f32(kPosThick, &h->thickness) || !R.f32(kPosEkv, &h->ekv) || !R.f32(kPosSx, &h->sx) ||
		!R.f32(kPosSy, &h->sy)) return 3;
	h->swapped = R.swap ? 1 : 0;
	if (h->nx <= 0 || h->ny <= 0 || h->nvar <= 0 || h->data_offset < (unsigned)kPosData) return 4;
	return 0;
}

int read_data(Reader& R, const JMSSliHeader& h, float* pgr)
{
	const size_t nf = (size_t)2 * h.nx * h.ny * h.nvar;
	if (std::fseek(R.f, (long)h.data_offset, SEEK_SET) != 0) return 5;
	if (std::fread(pgr, sizeof(float), nf, R.f) != nf) return 5;
	if (R.swap) {
		uint32_t* p = reinterpret_cast<uint32_t*>(pgr);
		for (size_t i = 0; i < nf; i++) p[i] = bswap32(p[i]);
	}
	return 0;
}
} // namespace

extern "C" {

int JMS_SliReadHeader(const char* path, JMSSliHeader* hdr)
{
	if (!path || !hdr) return 1;
	Reader R;
	return read_header(R, path, hdr);
}

int JMS_SliReadData(const char* path, float* pgr)
{
	if (!path || !pgr) return 1;
	Reader R;
	JMSSliHeader h;
	int e = read_header(R, path, &h);
	if (e) return e;
	return read_data(R, h, pgr);
}

int JMS_SliWrite(const char* path, const JMSSliHeader* hdr, const float* pgr)
{
	if (!path || !hdr || !pgr || hdr->nx <= 0 || hdr->ny <= 0 || hdr->nvar <= 0) return 1;
	std::vector<unsigned char> head(kPosData, 0);
	auto put = [&](long pos, const void* v) { std::memcpy(&head[pos], v, 4); };
	const uint32_t nx = (uint32_t)hdr->nx, ny = (uint32_t)hdr->ny, nvar = (uint32_t)hdr->nvar;
	const uint32_t content = (uint32_t)hdr->content, doff = (uint32_t)kPosData, toff = (uint32_t)kPosTab;
	put(kPosNx, &nx);
	put(kPosNy, &ny);
	std::memcpy(&head[kPosTitle], hdr->title, 40);
	put(kPosVer, &kVerWrite);
	put(kPosNvar, &nvar);
	put(kPosContent, &content);
	put(kPosAltOffset, &doff);
	put(kPosTabOffset, &toff);
	put(kPosThick, &hdr->thickness);
	put(kPosEkv, &hdr->ekv);
	put(kPosSx, &hdr->sx);
	put(kPosSy, &hdr->sy);
	// the atom table at 0x1100 stays empty (zero atom types)
	std::FILE* f = std::fopen(path, "wb");
	if (!f) return 2;
	const size_t nf = (size_t)2 * nx * ny * nvar;
	const bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size() &&
		std::fwrite(pgr, sizeof(float), nf, f) == nf;
	return (std::fclose(f) == 0 && ok) ? 0 : 6;
}

} // extern "C"
