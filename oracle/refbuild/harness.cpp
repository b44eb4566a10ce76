// Drives the reference's own unstructured NS/SA solver (compiled from its
// sources into oracle/_ref/libphref.a) on a grid that is built in memory, and
// dumps its arrays as raw binary goldens.  Test infrastructure only.
//
// The set-up follows the reference's start-up sequence for a one-zone,
// one-rank steady run:
//   RunPHengLEI        Main/src/CFDSimulation.cpp:19-47
//   Simulation::RunCFD Main/src/Simulation.cpp:205-277
//   grid ingestion     API/PreProcess/src/Pre_HDF5File.cpp:891-908, 1753-1940,
//                      2128-2235 (the HDF5 reads replaced by in-memory arrays)
//   outer loop         Main/src/Simulation.cpp:1292-1327, 1190-1237, 1527-1559
//
// usage: ref_harness MESH RUNDIR OUTDIR NSTEPS [STATE] [name:rows:cols ...]
//   MESH   binary mesh (format written by phenlei_b200/mesh.py:write_mesh), or
//          a comma-separated list of meshes, one zone each, all on this rank;
//          a zone's MESH.itf file, when present, holds its interface data as
//          the reference's grid files do (IO_HDF5Read::ReadInterfaceInfo,
//          Pre_HDF5File.cpp:1366-1401): int64 nIFace, then interFace2ZoneID,
//          interFace2InterFaceID and interFace2BoundaryFace (int32 each).
//          Several zones write their dumps to OUTDIR/zone<i>/.
//   RUNDIR directory holding bin/key.hypara and the case files
//   STATE  optional binary primitive state (nEq x nTotalCell doubles, then
//          optionally nTurb x nTotalCell) that replaces the initial field; "-"
//          for none; one file per zone, comma-separated
//   name:rows:cols  grid data arrays to dump after the last step (rows=0 means
//          a 1-D array of cols values)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <unistd.h>
#include <sys/stat.h>
#include <execinfo.h>
#include <signal.h>
#include <sstream>
#include <fstream>
#include <iomanip>
#include <map>
#include <set>
#include <list>
#include <deque>
#include <queue>
#include <stack>
#include <algorithm>
#include <functional>
#include <memory>
#include <cmath>
#include <complex>
#include <numeric>
#include <iterator>
#include <utility>
#include <limits>
#include <bitset>
#include <unordered_map>
#include <unordered_set>
#include <array>
#include <tuple>
#include <valarray>
#include <random>
#include <mutex>
#include <thread>
#define private public
#define protected public
#include "PHMpi.h"
#include "GlobalDataBase.h"
#include "Region.h"
#include "Zone.h"
#include "Geo_UnstructGrid.h"
#include "Geo_UnstructBC.h"
#include "Geo_SimpleBC.h"
#include "Geo_SimpleVC.h"
#include "NSSolverUnstruct.h"
#include "TurbSolverUnstr.h"
#include "Controller.h"
#include "PHIO.h"
#include "Constants.h"
#include "Glb_Dimension.h"
#include "Pre_WalldistCompute.h"
#include "AleManager.h"
#include "TK_Time.h"
#undef private
#undef protected

// The parameter self-check of the reference (ParametersSelfCheckForCFD) has
// internal linkage; its translation unit is compiled here, in place.
#include PHX_REF_CFDSIMULATION

using namespace PHSPACE;

namespace
{
struct MeshFile
{
    long long nNode, nFace, nCell, nBFace, nF2N, nC2N, nRegion;
    std::vector<double> x, y, z;
    std::vector<int> nodePerFace, face2node, left, right, nodePerCell, cell2node, bfaceRegion;
    std::vector<int> regionType;
    std::vector<std::string> regionName;
};

static bool g_trace = getenv("PHX_HARNESS_TRACE") != nullptr;
#define STAGE(msg) do { if (g_trace) { fprintf(stderr, "[harness] %s\n", msg); fflush(stderr); } } while (0)

void OnFault(int sig)
{
    void *frames[64];
    int n = backtrace(frames, 64);
    fprintf(stderr, "ref_harness: signal %d\n", sig);
    backtrace_symbols_fd(frames, n, 2);
    _exit(3);
}

void Die(const char *msg)
{
    fprintf(stderr, "ref_harness: %s\n", msg);
    exit(2);
}

template <class T>
void ReadVec(FILE *f, std::vector<T> &v, long long n)
{
    v.resize(n);
    if (n && fread(v.data(), sizeof(T), n, f) != (size_t)n) Die("short read");
}

MeshFile ReadMesh(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) Die("cannot open mesh");
    char magic[8];
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "PHXMESH1", 8)) Die("bad mesh magic");
    MeshFile m;
    long long h[7];
    if (fread(h, sizeof(long long), 7, f) != 7) Die("short header");
    m.nNode = h[0]; m.nFace = h[1]; m.nCell = h[2]; m.nBFace = h[3];
    m.nF2N = h[4]; m.nC2N = h[5]; m.nRegion = h[6];
    ReadVec(f, m.x, m.nNode); ReadVec(f, m.y, m.nNode); ReadVec(f, m.z, m.nNode);
    ReadVec(f, m.nodePerFace, m.nFace); ReadVec(f, m.face2node, m.nF2N);
    ReadVec(f, m.left, m.nFace); ReadVec(f, m.right, m.nFace);
    ReadVec(f, m.nodePerCell, m.nCell); ReadVec(f, m.cell2node, m.nC2N);
    ReadVec(f, m.bfaceRegion, m.nBFace);
    for (long long r = 0; r < m.nRegion; ++r)
    {
        int t, len;
        if (fread(&t, 4, 1, f) != 1 || fread(&len, 4, 1, f) != 1) Die("short region");
        std::string name(len, ' ');
        if (fread(&name[0], 1, len, f) != (size_t)len) Die("short region name");
        m.regionType.push_back(t);
        m.regionName.push_back(name);
    }
    fclose(f);
    return m;
}

struct ItfFile
{
    long long nIFace = 0;
    std::vector<int> zoneID, interFaceID, boundaryFace;
};

ItfFile ReadItf(const std::string &path)
{
    ItfFile itf;
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return itf;
    if (fread(&itf.nIFace, sizeof(long long), 1, f) != 1) Die("short interface file");
    ReadVec(f, itf.zoneID, itf.nIFace);
    ReadVec(f, itf.interFaceID, itf.nIFace);
    ReadVec(f, itf.boundaryFace, itf.nIFace);
    fclose(f);
    return itf;
}

std::vector<std::string> SplitList(const std::string &s)
{
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ',')) out.push_back(item);
    return out;
}

template <class T>
T *Dup(const std::vector<T> &v)
{
    T *p = new T[v.size() ? v.size() : 1];
    if (!v.empty()) memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

// Mirrors IO_HDF5Read::ReadUnstructGrid / ReadFaceTopology / ReadCellTopology /
// ReadUnstrBCName (Pre_HDF5File.cpp:1753-1940) with the arrays taken from MESH.
UnstructGrid *BuildGrid(const MeshFile &m, int zoneIndex, const ItfFile &itf)
{
    GridID *index = new GridID(zoneIndex);
    UnstructGrid *grid = new UnstructGrid();
    grid->InitGrid(index, 0, PHSPACE::GetDim(), UNSTRUCTGRID);
    grid->SetIBlock(0);
    grid->SetNTotalNode((int)m.nNode);
    grid->SetNTotalFace((int)m.nFace);
    grid->SetNTotalCell((int)m.nCell);

    grid->SetX(Dup(m.x));
    grid->SetY(Dup(m.y));
    grid->SetZ(Dup(m.z));
    grid->RotateAboutAxis();
    grid->ComputeMinMaxBox();

    grid->SetNodeNumberOfEachFace(Dup(m.nodePerFace));
    grid->SetFace2Node(Dup(m.face2node));
    grid->SetLeftCellOfFace(Dup(m.left));
    grid->SetRightCellOfFace(Dup(m.right));
    grid->SetNBoundFace((int)m.nBFace);
    grid->SpecifyRightCellofBC();

    grid->SetInterfaceInfo(0);
    if (itf.nIFace > 0)
    {
        InterfaceInfo *info = new InterfaceInfo((int)itf.nIFace, grid);
        for (long long i = 0; i < itf.nIFace; ++i)
        {
            info->GetInterFace2ZoneID()[i] = itf.zoneID[i];
            info->GetInterFace2InterFaceID()[i] = itf.interFaceID[i];
            info->GetInterFace2BoundaryFace()[i] = itf.boundaryFace[i];
        }
        grid->SetInterfaceInfo(info);
    }
    grid->SetNodeNumberOfEachCell(Dup(m.nodePerCell));
    grid->SetCell2Node(Dup(m.cell2node));

    int nBoundFace = (int)m.nBFace;
    UnstructBCSet **bcr = new UnstructBCSet *[nBoundFace];
    for (int iFace = 0; iFace < nBoundFace; ++iFace)
    {
        int r = m.bfaceRegion[iFace];
        bcr[iFace] = new UnstructBCSet();
        bcr[iFace]->SetKey(m.regionType[r]);
        bcr[iFace]->SetBCName(m.regionName[r]);
    }
    grid->SetBCRecord(bcr);

    // Regions are numbered in name order, as std::set<string> orders them.
    std::vector<int> order((size_t)m.nRegion);
    for (int r = 0; r < (int)m.nRegion; ++r) order[r] = r;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return m.regionName[a] < m.regionName[b]; });
    grid->CreateUnstructBCSet((int)m.nRegion);
    UnstructBCSet *set = grid->GetUnstructBCSet();
    int *regionOfFace = new int[nBoundFace ? nBoundFace : 1];
    for (int k = 0; k < (int)m.nRegion; ++k)
    {
        int r = order[k];
        UnstructBC *bc = new UnstructBC(k);
        set->SetBCRegion(k, bc);
        bc->SetBCName(m.regionName[r]);
        bc->SetBCType(m.regionType[r]);
        for (int iFace = 0; iFace < nBoundFace; ++iFace)
        {
            if (m.bfaceRegion[iFace] == r)
            {
                regionOfFace[iFace] = k;
                bc->GetFaceIndex()->push_back(iFace);
            }
        }
    }
    set->SetBCFaceInfo(regionOfFace);
    return grid;
}

// Every zone on this rank (processor 0), as a one-rank run of a partitioned
// grid lays them out.
void SetLayout(int nZones)
{
    PHMPI::SetNumberOfGlobalZones(nZones);
    PHMPI::CreateZoneProcessorIDDump(nZones);
    PHMPI::CreateZoneProcessorID(nZones);
    PHMPI::CreateZoneGridID(nZones);
    PHMPI::CreateZoneGridType(nZones);
    PHMPI::CreateZoneFileID(nZones);
    for (int z = 0; z < nZones; ++z)
    {
        PHMPI::GetZoneProcessorID()[z] = 0;
        PHMPI::GetZoneProcessorIDForGrid()[z] = -1;
        PHMPI::GetZoneGridType()[z] = UNSTRUCTGRID;
        PHMPI::GetZoneGridID()[z] = z;
        PHMPI::GetZoneFileID()[z] = 0;
        PHMPI::GetZoneProcessorIDDump()[z] = 0;
    }
    int sysGridType = UNSTRUCTGRID;
    GlobalDataBase::UpdateData("sys_gridtype", &sysGridType, PHINT, 1);
}

void WriteRaw(const std::string &path, const double *p, size_t n)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) Die("cannot write output");
    fwrite(p, sizeof(double), n, f);
    fclose(f);
}
}  // namespace

int main(int argc, char **argv)
{
    if (argc < 5) Die("usage: ref_harness MESH RUNDIR OUTDIR NSTEPS [STATE] [name:rows:cols ...]");
    signal(SIGSEGV, OnFault);
    signal(SIGBUS, OnFault);
    const std::vector<std::string> meshPaths = SplitList(argv[1]);
    const int nZones = (int)meshPaths.size();
    if (nZones < 1) Die("no mesh");
    std::vector<MeshFile> meshes;
    std::vector<ItfFile> itfs;
    for (const std::string &mp : meshPaths)
    {
        meshes.push_back(ReadMesh(mp.c_str()));
        itfs.push_back(ReadItf(mp + ".itf"));
    }
    std::string outdir = argv[3];
    int nSteps = atoi(argv[4]);
    if (chdir(argv[2]) != 0) Die("cannot chdir to RUNDIR");

    STAGE("init");
    PHMPI::Initialization();
    ReadControlParameters();
    STAGE("params read");
    CompleteParamInfo();
    ControlParametersPreliminarySelfCheck();
    SetDim(GlobalDataBase::GetIntParaFromDB("ndim"));

    STAGE("self check done");
    Region *region = new Region();
    SetLayout(nZones);
    std::vector<UnstructGrid *> grids;
    for (int z = 0; z < nZones; ++z)
    {
        // IO_HDF5Read::CreateZones (Pre_HDF5File.cpp:2206-2235)
        UnstructGrid *grid = BuildGrid(meshes[z], z, itfs[z]);
        grid->GetGridID()->SetLocalIndex(PHMPI::GetNumberofLocalZones());
        Zone *zone = new Zone(z);
        zone->AddGridAndCopyZonePara(grid);
        zone->AddGridToGlobal(z);
        region->AddZone(zone);
        grids.push_back(grid);
    }
    STAGE("grid built");
    GlobalBoundaryCondition::ReadGlobalBoundaryCondition();
    region->AllocateOversetGrid();

    STAGE("bc read");
    region->UpdateAllZonesPara();
    STAGE("zone para");
    region->InitGeometry();
    STAGE("geometry");
    region->SwapGeometry();

    // Simulation::DefineAndCreateSolvers (Simulation.cpp:977-1188), every zone.
    STAGE("swap geometry");
    InitGlobalValuesOfAllZones();
    for (int z = 0; z < nZones; ++z)
    {
        Zone *zone = region->GetZone(z);
        std::vector<PHSolver *> solvers;
        PHSolver *ns = new NSSolverUnstruct();
        ns->SetName("NSSolverUnstruct");
        ns->SetKey(DENSITY_BASED_SOLVER);
        solvers.push_back(ns);
        int viscousType = GlobalDataBase::GetIntParaFromDB("viscousType");
        if (viscousType > LAMINAR)
        {
            PHSolver *turb = new TurbSolverUnstr();
            turb->SetName("TurbSolverUnstr");
            turb->SetKey(DENSITY_BASED_SOLVER);
            solvers.push_back(turb);
        }
        for (size_t i = 0; i < solvers.size(); ++i)
        {
            solvers[i]->SetGeometry(zone->GetGeometry());
            solvers[i]->SetIndex((int)i);
            zone->AddSolver(solvers[i]);
        }
        int maxNumOfSolver = (int)solvers.size();
        GlobalDataBase::UpdateData("maxNumOfSolver", &maxNumOfSolver, PHINT, 1);
    }
    STAGE("solvers");
    region->ReSetBoundaryConditionByGlobalBC();
    GlobalVolumeCondition::ReadGlobalVolumeCondition();
    GlobalVolumeCondition::SetVCDataByGlobalVC();

    // GenerateWalldist (Pre_WalldistCompute.cpp:5296-5342) without the file write.
    {
        int viscousType = GlobalDataBase::GetIntParaFromDB("viscousType");
        if (viscousType != INVISCID)
        {
            AllocateWalldist();
            // PHX_REF_WALLDIST names a file of nTotalCell doubles that replaces
            // the reference's wall-distance search (its set-up cost grows with
            // cells x wall faces); only the timing runs use it
            const char *wdFile = getenv("PHX_REF_WALLDIST");
            if (wdFile && *wdFile)
            {
                const std::vector<std::string> wdPaths = SplitList(wdFile);
                if ((int)wdPaths.size() != nZones) Die("PHX_REF_WALLDIST needs one file per zone");
                for (int z = 0; z < nZones; ++z)
                {
                    FILE *wf = fopen(wdPaths[z].c_str(), "rb");
                    if (!wf) Die("cannot open PHX_REF_WALLDIST");
                    RDouble *wd = grids[z]->GetWallDist();
                    const size_t nread = fread(wd, sizeof(RDouble), grids[z]->GetNTotalCell(), wf);
                    fclose(wf);
                    if ((int)nread != grids[z]->GetNTotalCell()) Die("short PHX_REF_WALLDIST file");
                }
            }
            else
            {
                ComputeWalldist();
            }
        }
        if (viscousType > LAMINAR) WalldistStatics();
        int flowInitMethod = GlobalDataBase::GetIntParaFromDB("flowInitMethod");
        if (viscousType != INVISCID && flowInitMethod > 0) CompMaxBoundaryLayerWalldist();
    }

    STAGE("walldist");
    int nSolver = GlobalDataBase::GetIntParaFromDB("maxNumOfSolver");
    for (int iSolver = 0; iSolver < nSolver; ++iSolver)
    {
        Controller *controller = new Controller(iSolver, region);
        controller->Initialize(iSolver);
        delete controller;
    }
    STAGE("initialized");
    CreateAleManager();

    int nl = GlobalDataBase::GetIntParaFromDB("nl");
    int nTurb = (nSolver > 1) ? GlobalDataBase::GetIntParaFromDB("n_turb") : 0;

    if (argc > 5 && strcmp(argv[5], "-") != 0)
    {
        const std::vector<std::string> statePaths = SplitList(argv[5]);
        if ((int)statePaths.size() != nZones) Die("STATE needs one file per zone");
        for (int z = 0; z < nZones; ++z)
        {
            UnstructGrid *grid = grids[z];
            const int nTotalCell = grid->GetNTotalCell();
            FILE *f = fopen(statePaths[z].c_str(), "rb");
            if (!f) Die("cannot open STATE");
            RDouble **q = reinterpret_cast<RDouble **>(grid->GetDataPtr("q"));
            for (int m = 0; m < nl; ++m)
                if (fread(q[m], sizeof(double), nTotalCell, f) != (size_t)nTotalCell) Die("short STATE");
            if (nTurb)
            {
                RDouble **qt = reinterpret_cast<RDouble **>(grid->GetDataPtr("q_turb"));
                for (int m = 0; m < nTurb; ++m)
                {
                    size_t got = fread(qt[m], sizeof(double), nTotalCell, f);
                    if (got != 0 && got != (size_t)nTotalCell) Die("short STATE (turb)");
                }
            }
            fclose(f);
            // GG-node gradients read node values that the solver forms at
            // initialisation (NSSolver::InitDependentVariables, NSSolver.cpp:757-790,
            // then Controller::Initialize's ModifyNodeValue) and in each PostSolve;
            // a loaded state gets them the way an initialisation from a restart does.
            if (GlobalDataBase::GetStrParaFromDB("gradientName") == "ggnode")
            {
                NSSolverUnstruct *ns = static_cast<NSSolverUnstruct *>(GlobalSolvers::GetSolver(z, 0));
                ns->InitDependentVariables();
                ns->ModifyNodeValue(grid);
                if (nTurb)
                {
                    // the SA solver's node values of nu~ (TurbSolver::InitDependentVariables,
                    // TurbSolver.cpp:46-56, then ModifyQTurbNodeValue)
                    TurbSolverUnstr *turb = static_cast<TurbSolverUnstr *>(GlobalSolvers::GetSolver(z, 1));
                    turb->InitDependentVariables();
                    turb->ModifyQTurbNodeValue(grid);
                }
            }
        }
        // Controller::Initialize ends with the interface communication of
        // every zone (Controller.cpp:153-172); the loaded state takes its place
        // here, so the interface ghosts receive the neighbours' loaded cells
        if (nZones > 1)
            for (int iSolver = 0; iSolver < nSolver; ++iSolver)
                for (int z = 0; z < nZones; ++z) GlobalSolvers::GetSolver(z, iSolver)->CommunicationInterfaceData();
    }

    // Outer loop: Simulation::SolveSimulation / SolveOneOuterStep without the
    // visual-file output of Simulation::PostSolve.
    int outIterStep = GlobalDataBase::GetIntParaFromDB("outnstep");
    std::vector<double> resHist;
    // wall time of the iteration loop alone (set-up and output excluded): the
    // reference's own throughput on this host, written to iter_seconds.bin
    const auto loopStart = std::chrono::steady_clock::now();
    for (int step = 0; step < nSteps; ++step)
    {
        ++outIterStep;
        GlobalDataBase::UpdateData("outnstep", &outIterStep, PHINT, 1);
        int newIterStep = GlobalDataBase::GetIntParaFromDB("newnstep") + 1;
        GlobalDataBase::UpdateData("newnstep", &newIterStep, PHINT, 1);

        int isInIniting = GlobalDataBase::GetIntParaFromDB("isInIniting");
        int flowInitStep = GlobalDataBase::GetIntParaFromDB("flowInitStep");
        if (isInIniting == 1 && ((flowInitStep > 0 && outIterStep > flowInitStep) || flowInitStep == 0))
        {
            isInIniting = 0;
            GlobalDataBase::UpdateData("isInIniting", &isInIniting, PHINT, 1);
        }

        int turbInterval = GlobalDataBase::GetIntParaFromDB("turbInterval");
        for (int iSolver = 0; iSolver < nSolver; ++iSolver)
        {
            if (iSolver != NS_SOLVER && (outIterStep % turbInterval != 0)) break;
            Controller *controller = new Controller(iSolver, region);
            STAGE("solve");
            controller->SolveSteadyField();
            STAGE("post");
            controller->PostSolve();
            delete controller;
        }

        // Residual monitor of NS equation 0 (Residual.cpp:184-224 definition),
        // summed over the zones (PH_AllReduce)
        double s = 0.0;
        long long n = 0;
        for (int z = 0; z < nZones; ++z)
        {
            RDouble **res = reinterpret_cast<RDouble **>(grids[z]->GetDataPtr("res"));
            const int nc = grids[z]->GetNTotalCell();
            for (int c = 0; c < nc; ++c) s += res[0][c] * res[0][c];
            n += nc;
        }
        resHist.push_back(sqrt(s / n));
    }
    const double loopSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - loopStart).count();
    WriteRaw(outdir + "/iter_seconds.bin", &loopSeconds, 1);
    WriteRaw(outdir + "/res_hist.bin", resHist.data(), resHist.size());

    for (int z = 0; z < nZones; ++z)
    {
        UnstructGrid *grid = grids[z];
        const int nTotalCell = grid->GetNTotalCell();
        const int nTotal = nTotalCell + grid->GetNBoundFace();
        std::string outdir = argv[3];
        if (nZones > 1)
        {
            outdir += "/zone" + std::to_string(z);
            mkdir(outdir.c_str(), 0755);
        }
        for (int a = 6; a < argc; ++a)
        {
            char name[256];
            int rows = 0, cols = 0;
            if (sscanf(argv[a], "%255[^:]:%d:%d", name, &rows, &cols) != 3) Die("bad dump spec");
            void *p = grid->GetDataPtr(name);
            if (!p)
            {
                fprintf(stderr, "ref_harness: no array %s\n", name);
                continue;
            }
            std::vector<double> buf;
            if (rows == 0)
            {
                buf.assign((RDouble *)p, (RDouble *)p + cols);
            }
            else
            {
                RDouble **pp = reinterpret_cast<RDouble **>(p);
                for (int r = 0; r < rows; ++r) buf.insert(buf.end(), pp[r], pp[r] + cols);
            }
            WriteRaw(outdir + "/" + name + ".bin", buf.data(), buf.size());
        }
        // Geometry as the reference computed it.
        WriteRaw(outdir + "/xfn.bin", grid->GetFaceNormalX(), grid->GetNTotalFace());
        WriteRaw(outdir + "/yfn.bin", grid->GetFaceNormalY(), grid->GetNTotalFace());
        WriteRaw(outdir + "/zfn.bin", grid->GetFaceNormalZ(), grid->GetNTotalFace());
        WriteRaw(outdir + "/area.bin", grid->GetFaceArea(), grid->GetNTotalFace());
        WriteRaw(outdir + "/xfc.bin", grid->GetFaceCenterX(), grid->GetNTotalFace());
        WriteRaw(outdir + "/yfc.bin", grid->GetFaceCenterY(), grid->GetNTotalFace());
        WriteRaw(outdir + "/zfc.bin", grid->GetFaceCenterZ(), grid->GetNTotalFace());
        WriteRaw(outdir + "/xcc.bin", grid->GetCellCenterX(), nTotal);
        WriteRaw(outdir + "/ycc.bin", grid->GetCellCenterY(), nTotal);
        WriteRaw(outdir + "/zcc.bin", grid->GetCellCenterZ(), nTotal);
        WriteRaw(outdir + "/vol.bin", grid->GetCellVolume(), nTotal);
        if (grid->GetWallDist()) WriteRaw(outdir + "/walldist.bin", grid->GetWallDist(), nTotalCell);
        // Wall force sums of NSSolverUnstruct::AirForceCoefParts (all parts): CA_f CA_p
        // CN_f CN_p CZ_f CZ_p cpx cpy cpz Cl_f Cl_p Cn_f Cn_p Cm_f Cm_p hingeMoment.
        {
            NSSolverUnstruct *ns = static_cast<NSSolverUnstruct *>(GlobalSolvers::GetSolver(z, 0));
            ActionKey *ak = new ActionKey();
            ak->level = 0;
            ns->AirForceCoefParts(ak, -1);
            DataContainer *cd = ak->GetData();
            cd->MoveToBegin();
            std::vector<RDouble> f(16, 0.0);
            for (int k = 0; k < 16; ++k) cd->Read(&f[k], sizeof(RDouble));
            WriteRaw(outdir + "/forces.bin", f.data(), f.size());
            delete ak;
        }
    }
    fprintf(stdout, "ref_harness: done %d steps, %d zone(s), zone 0 nTotalCell=%d nBoundFace=%d\n", nSteps, nZones,
            grids[0]->GetNTotalCell(), grids[0]->GetNBoundFace());
    return 0;
}
