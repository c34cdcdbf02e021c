// restir_struct_size: the byte size of every public struct of the C ABI, so
// that a binding in another language can check its copies of the layouts.
#include "../../include/restir_cache.h"
#include "../../include/restir_display.h"
#include "../../include/restir_frame.h"
#include "../../include/restir_host.h"

#include <cstring>

extern "C" uint64_t restir_struct_size(const char* name)
{
	if (name == nullptr)
	{
		return 0;
	}
	struct Entry
	{
		const char* name;
		uint64_t bytes;
	};
	static const Entry entries[] = {
		{ "RestirBatchTuning", sizeof(RestirBatchTuning) }, { "RestirBvhDesc", sizeof(RestirBvhDesc) },
		{ "RestirCacheConfig", sizeof(RestirCacheConfig) }, { "RestirCacheLayout", sizeof(RestirCacheLayout) },
		{ "RestirCacheScalars", sizeof(RestirCacheScalars) }, { "RestirDiReservoirs", sizeof(RestirDiReservoirs) },
		{ "RestirDisplayParams", sizeof(RestirDisplayParams) }, { "RestirFrameInput", sizeof(RestirFrameInput) },
		{ "RestirFramePlan", sizeof(RestirFramePlan) }, { "RestirFrameState", sizeof(RestirFrameState) },
		{ "RestirGBuffer", sizeof(RestirGBuffer) }, { "RestirGiHistory", sizeof(RestirGiHistory) },
		{ "RestirGiReservoirs", sizeof(RestirGiReservoirs) }, { "RestirLightsDesc", sizeof(RestirLightsDesc) },
		{ "RestirMeshDesc", sizeof(RestirMeshDesc) }, { "RestirMetrics", sizeof(RestirMetrics) },
		{ "RestirParams", sizeof(RestirParams) }, { "RestirScene", sizeof(RestirScene) },
		{ "RestirSettings", sizeof(RestirSettings) },
	};
	for (const Entry& e : entries)
	{
		if (std::strcmp(e.name, name) == 0)
		{
			return e.bytes;
		}
	}
	return 0;
}
